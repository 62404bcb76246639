"""Device and memory configuration (paces/config/_dev_conf.py:5-71).

One GPU holds everything: the basis keys, the Hamiltonian table and the amplitudes live
on the same device.  The reference's optional split of the lookup tables and the vectors
over two GPUs and its managed-memory pool are not offered (a B200 holds 180 GB).
"""

import torch


class Device:
    """A CUDA device usable as a context manager (`with devices.vector_dev:`)."""

    def __init__(self, index=0):
        self.id = int(index)
        self._ctx = None

    def __eq__(self, other):
        if isinstance(other, Device):
            return other.id == self.id
        if isinstance(other, torch.device):
            return other.type == "cuda" and (other.index or 0) == self.id
        return NotImplemented

    def __hash__(self):
        return hash(("cuda", self.id))

    def __enter__(self):
        if torch.cuda.is_available():
            self._ctx = torch.cuda.device(self.id)
            self._ctx.__enter__()
        return self

    def __exit__(self, *exc):
        if self._ctx is not None:
            self._ctx.__exit__(*exc)
            self._ctx = None
        return False

    @property
    def torch(self):
        return torch.device("cuda", self.id)

    def __repr__(self):
        return f"<CUDA Device {self.id}>"


class MemoryPool:
    """Reports PyTorch's caching allocator (the reference reports CuPy's pool)."""

    def __init__(self, device):
        self.device = device

    def used_bytes(self):
        return torch.cuda.memory_allocated(self.device.id) if torch.cuda.is_available() else 0

    def free_all_blocks(self):
        if torch.cuda.is_available():
            torch.cuda.empty_cache()


class DeviceConfig:
    """Placeholder until `configure` is called (paces/config/_dev_conf.py:5-27)."""

    def __init__(self):
        self.whoami_dev = None
        self.vector_dev = None
        self.mempool = None
        self.split = False
        self.desc_str = ""
        self.configure_called = False

    def _print_and_save(self, s):
        print(s)
        self.desc_str += s + "\n"

    def configure(self, whoami_device_id=0, vector_device_id=0, unified_memory_bytes=None):
        """Select the GPU (paces/config/_dev_conf.py:29-71).

        whoami_device_id and vector_device_id must name the same GPU, and
        unified_memory_bytes must be None: the two-GPU split and the managed-memory pool
        are not part of this implementation.
        """
        if whoami_device_id != vector_device_id:
            raise NotImplementedError("the basis and the vectors live on one GPU; "
                                      "whoami_device_id must equal vector_device_id")
        if unified_memory_bytes is not None:
            raise NotImplementedError("unified (managed) memory is not supported; "
                                      "leave unified_memory_bytes=None")
        print("######### CUDA device setup: #########")
        self.desc_str += "### CUDA device setup:\n"
        self.whoami_dev = Device(whoami_device_id)
        self.vector_dev = self.whoami_dev
        self.split = False
        self._print_and_save("    Using one GPU.")
        self.mempool = MemoryPool(self.vector_dev)
        self._print_and_save("    Using default (GPU-based) memory pool.")
        self.configure_called = True
        print("#########    end of setup    #########\n")
        self.desc_str += "\n"
