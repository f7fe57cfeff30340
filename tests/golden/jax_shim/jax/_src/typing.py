import numpy as _np
Array = _np.ndarray
ArrayLike = _np.ndarray
