"""`cupy.cuda.memory` stub for the CPU stand-in (test infrastructure)."""


def malloc_managed(size):
    raise NotImplementedError("the CPU stand-in has no managed memory")
