"""DOP853 orbit integration on the device."""


def orbit(*args, **kwargs):
    raise NotImplementedError
