class _Theme:
    pass


global_theme = _Theme()
