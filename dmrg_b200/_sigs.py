"""ctypes signatures of the C entry points beyond the matvec/operator core (see include/heff.h)."""


def declare(L, sig):
    return None
