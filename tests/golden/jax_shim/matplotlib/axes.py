def __getattr__(name):
    return object
