"""No-op plotting stub (fixtures never plot)."""
rcParams = {}


def use(*args, **kwargs):
    pass
