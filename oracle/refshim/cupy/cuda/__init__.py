"""Device/stream/memory stubs of `cupy.cuda` for the CPU stand-in (test infrastructure)."""

from . import memory  # noqa: F401


class Device:
    """Every device is the host.  NumPy 2 arrays report `.device == "cpu"`."""

    def __init__(self, device_id=0):
        if isinstance(device_id, Device):
            device_id = device_id.id
        self.id = int(device_id)

    def __eq__(self, other):
        if isinstance(other, Device):
            return other.id == self.id
        return other == "cpu"

    def __ne__(self, other):
        return not self.__eq__(other)

    def __hash__(self):
        return hash(("cpu-device", self.id))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def __repr__(self):
        return f"<CUDA Device {self.id} (CPU stand-in)>"

    def synchronize(self):
        pass

    @property
    def mem_info(self):
        return (0, 0)


class Stream:
    def __init__(self, *args, **kwargs):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def synchronize(self):
        pass


class MemoryPool:
    def __init__(self, *args, **kwargs):
        pass

    def set_limit(self, size=None):
        pass

    def malloc(self, size):
        raise NotImplementedError("the CPU stand-in has no device memory")

    def used_bytes(self):
        return 0

    def free_all_blocks(self):
        pass


def set_allocator(*args, **kwargs):
    pass
