"""spin_colour_kernel_b200: the colour-class Metropolis sweep of spin-colour-kernel on NVIDIA B200.

Host side (Python): crystals and bond tables, linear colourings, systems (the reference's system description),
the lowering of a system to the C descriptor and the host-built acceptance tables, and a `Sampler` with the
reference's interface. Device side: hand-written sm_100a CUDA in csrc/, built into libsckb200.so and called
through the C ABI of include/sck.h.
"""

from . import colouring, crystals, system  # noqa: F401

__all__ = ["colouring", "crystals", "system", "Sampler"]


def __getattr__(name):
    if name == "Sampler":
        from .sampler import Sampler
        return Sampler
    raise AttributeError(name)
