"""Sharding a spiking network over ranks by post-synaptic neurons.

Rank r of W owns a contiguous, 32-aligned slice of every population
(owned_range) and the incoming synapses of its neurons: it updates only its
slice, transmits only onto it, and the plastic synapses it holds are those of
its post neurons (both STDP sides stay local). After every step the ranks
exchange the spike bitmap words of their slices (an all-gather of one chunk
of words per rank), so that every rank sees all spikes of the step before its
next transmission. The reference runs one process per network and has no
multi-GPU path; this follows the row sharding of the 1e9-synapse network.
"""
from __future__ import annotations

import numpy as np


def chunk_words(n: int, world: int) -> int:
    """Bitmap words per rank (the last rank may own fewer neurons)."""
    words = -(-n // 32)
    return max(1, -(-words // world))


def owned_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) of the neurons of an n-neuron population owned by `rank`."""
    c = chunk_words(n, world)
    return min(n, 32 * c * rank), min(n, 32 * c * (rank + 1))


class Exchange:
    """All-gather of per-rank chunks of spike bitmap words through
    torch.distributed (gloo: host tensors; nccl: device tensors)."""

    def __init__(self, rank: int, world: int, group=None):
        import torch.distributed as dist
        self.rank, self.world, self.group = rank, world, group
        self.dist = dist
        backend = dist.get_backend(group) if dist.is_initialized() else None
        if backend is None:
            raise RuntimeError("sharded networks need an initialised torch.distributed process group")
        self.device = "cuda" if backend == "nccl" else "cpu"

    def all_gather_device(self, native, array: str, chunk: int):
        """In-place all-gather of `chunk` 32-bit words per rank in the device
        array `array` of the network (rank r's words at r * chunk): NCCL reads
        this rank's chunk and writes the others' into the same buffer. The
        collective waits for the work already queued on the network's stream
        and the stream waits for it, so the next step's kernels see every
        rank's spikes without a host synchronisation."""
        import torch
        ptr, nbytes = native.device_ptr(array), native.nbytes(array)
        if nbytes < 4 * chunk * self.world:
            raise RuntimeError(f"{array}: {nbytes} bytes cannot hold {self.world} chunks of {chunk} words")

        class _View:                      # the array's memory seen by torch, no copy
            __cuda_array_interface__ = {"shape": (chunk * self.world,), "typestr": "<i4",
                                        "data": (ptr, False), "version": 3, "strides": None}
        full = torch.as_tensor(_View(), device="cuda")
        stream = torch.cuda.ExternalStream(native.stream())
        with torch.cuda.stream(stream):
            self.dist.all_gather_into_tensor(full, full[self.rank * chunk:(self.rank + 1) * chunk],
                                             group=self.group)

    def all_gather(self, local: np.ndarray) -> np.ndarray:
        import torch
        t = torch.from_numpy(np.ascontiguousarray(local).view(np.int32)).to(self.device)
        parts = [torch.empty_like(t) for _ in range(self.world)]
        self.dist.all_gather(parts, t, group=self.group)
        return torch.cat(parts).cpu().numpy().view(np.uint32)
