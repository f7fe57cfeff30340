class GradientDescent:
    pass


class OptaxSolver:
    pass


class NonlinearCG:
    pass
