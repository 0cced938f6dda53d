"""Batched weighted sums of one block-sparse matrix on the tensor cores.

Many instances of a rate-coded network that share their weights (a
parameter or input sweep) need, per projection and step, Y = X W^T for a
batch of rate vectors X (batch x n_pre) instead of one weighted sum per
instance (the reference's per-instance BSR kernel,
ANNarchy/generator/Projection/CUDA/BSR.py:296, run once per copy). With the
weights stored as dense 64 x 64 bfloat16 blocks, every block is a
64 x 64 x batch matrix product: `BlockSparseBatch` runs them with
tcgen05.mma (accumulators in tensor memory, csrc/bsr_tc.cu) and, for
comparison, on the CUDA cores.

    bsb = BlockSparseBatch(w, batch=128)        # w: scipy (n_post, n_pre)
    y = bsb(x)                                  # x: (128, n_pre) -> (128, n_post)
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sp

from .core.backend import to_bf16, from_bf16
from .generator.formats import bsr_arrays
from .runtime import lib as L

TILE = 64


def canonical_tiles(values: np.ndarray) -> np.ndarray:
    """(n_tiles, rows, 64) tiles indexed [tile][row][k] -> the tcgen05
    canonical K-major layout without swizzle, flattened: element (r, k) of a
    tile at ((r//8)*8 + k//8)*64 + (r%8)*8 + k%8 (rows a multiple of 8)."""
    v = np.asarray(values)
    n, rows, k = v.shape
    v = v.reshape(n, rows // 8, 8, k // 8, 8)                # tile, row group, r, k group, k
    return np.ascontiguousarray(v.transpose(0, 1, 3, 2, 4)).reshape(-1)


def pack_x_reference(x: np.ndarray) -> np.ndarray:
    """Host restatement of anb_bsr_tc_pack_x: (batch, n_pre) float ->
    bfloat16 tiles (ceil(n_pre/64) tiles of batch x 64, canonical layout)."""
    batch, n_pre = x.shape
    nbc = -(-n_pre // TILE)
    xp = np.zeros((batch, nbc * TILE), dtype=np.float32)
    xp[:, :n_pre] = x
    tiles = xp.reshape(batch, nbc, TILE).transpose(1, 0, 2)    # bc, b, k
    return to_bf16(canonical_tiles(tiles))


def tc_shape(ctas_per_sm: int = 0, stages: int = 0, group: int = 0):
    """Launch shape of the tensor-core product for this process (0 = the
    automatic choice); see anb_bsr_spmm_tc_shape."""
    rc = L.load().anb_bsr_spmm_tc_shape(int(ctas_per_sm), int(stages), int(group))
    if rc != 0:
        raise ValueError(f"launch shape ({ctas_per_sm}, {stages}, {group}) out of range")


def tc_prefetch(blocks: int = 4):
    """L2 prefetch distance (blocks) of the tensor-core product's weight
    tiles for this process; see anb_bsr_spmm_tc_prefetch."""
    if L.load().anb_bsr_spmm_tc_prefetch(int(blocks)) != 0:
        raise ValueError(f"prefetch distance {blocks} out of range (0-64)")


class BlockSparseBatch:
    """Weights w (scipy sparse, n_post x n_pre) as 64 x 64 bfloat16 blocks on
    device `device`; calls compute y[b] = w @ x[b] for `batch` rate vectors
    (batch a multiple of 16, at most 256)."""

    def __init__(self, w, batch: int, device: int = 0):
        if batch % 16 or not 16 <= batch <= 256:
            raise ValueError("batch must be a multiple of 16 between 16 and 256")
        w = sp.csr_matrix(w)
        w.sort_indices()
        self.n_post, self.n_pre = w.shape
        self.batch = batch
        d = bsr_arrays(np.arange(self.n_post), w.indptr, w.indices, w.data, self.n_pre, TILE)
        vals = d["values"].reshape(-1, TILE, TILE).transpose(0, 2, 1)   # [block][row][k]
        self.n_blocks = int(d["n_blocks"])
        self.n_block_rows = int(d["n_block_rows"])
        self.n_bcols = -(-self.n_pre // TILE)
        self.tiles_host = to_bf16(canonical_tiles(vals))
        nat = self.nat = L.NativeNet(device)
        nat.initialize(1.0)
        nat.create("brow", d["block_row_ptr"].astype(np.int32))
        nat.create("bcol", d["block_col"].astype(np.int32))
        nat.create("tiles", self.tiles_host)
        nat.create_empty("x", np.float32, (batch, self.n_pre))
        nat.create_empty("xt", np.uint16, (self.n_bcols * batch * TILE,))
        nat.create("y", np.zeros((batch, self.n_post), np.float32))
        nat.create("kerr", np.zeros(1, np.int32))
        self._p = {n: nat.device_ptr(n) for n in ("brow", "bcol", "tiles", "x", "xt", "y", "kerr")}
        # the products run on the stream of the arrays' copies
        self._stream = C.c_void_p(nat.stream())

    def _check(self, name, rc):
        if rc != 0:
            raise L.BackendError(name, rc, "bad argument" if rc == 2 else "CUDA error")

    def load(self, x: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32)
        if x.shape != (self.batch, self.n_pre):
            raise ValueError(f"x must be ({self.batch}, {self.n_pre})")
        self.nat.write("x", x)
        self.nat.zero("y")

    def pack(self):
        """Convert the loaded rates to bfloat16 tiles on the device (no sync)."""
        lib, p = L.load(), self._p
        self._check("anb_bsr_tc_pack_x", lib.anb_bsr_tc_pack_x(
            C.c_void_p(p["x"]), self.batch, self.n_pre, C.c_void_p(p["xt"]), self._stream))

    def product(self, engine: str = "tc"):
        """Add W x of the packed rates into y on the device (no sync)."""
        lib, p = L.load(), self._p
        if engine == "tc":
            self._check("anb_bsr_spmm_tc", lib.anb_bsr_spmm_tc(
                C.c_void_p(p["brow"]), C.c_void_p(p["bcol"]), C.c_void_p(p["tiles"]),
                self.n_block_rows, C.c_void_p(p["xt"]), self.batch, C.c_void_p(p["y"]),
                self.n_post, C.c_void_p(p["kerr"]), self._stream))
        elif engine == "simt":
            self._check("anb_bsr_spmm_simt", lib.anb_bsr_spmm_simt(
                C.c_void_p(p["brow"]), C.c_void_p(p["bcol"]), C.c_void_p(p["tiles"]),
                self.n_block_rows, C.c_void_p(p["xt"]), self.batch, C.c_void_p(p["y"]),
                self.n_post, self._stream))
        else:
            raise ValueError(engine)

    def run(self, engine: str = "tc"):
        """Pack the loaded rates and add W x into y on the device (no sync)."""
        if engine not in ("tc", "simt"):
            raise ValueError(engine)
        self.pack()
        self.product(engine)

    def result(self) -> np.ndarray:
        self.nat.synchronize()
        err = self.nat.read("kerr")
        if err[0]:
            raise L.BackendError("anb_bsr_spmm_tc", 5, f"device error code {int(err[0])}")
        return self.nat.read("y")

    def __call__(self, x: np.ndarray, engine: str = "tc") -> np.ndarray:
        self.load(x)
        self.run(engine)
        return self.result()

    def reference(self, x: np.ndarray) -> np.ndarray:
        """float64 product with the operands rounded to bfloat16 as the
        kernels see them (test oracle)."""
        wq = np.zeros((self.n_block_rows * TILE, self.n_bcols * TILE))
        d = from_bf16(self.tiles_host).reshape(-1, 8, 8, 8, 8).transpose(0, 1, 3, 2, 4)
        d = d.reshape(-1, TILE, TILE)                          # back to [block][row][k]
        brow = self.nat.read("brow")
        bcol = self.nat.read("bcol")
        for br in range(self.n_block_rows):
            for j in range(brow[br], brow[br + 1]):
                wq[br * TILE:(br + 1) * TILE, bcol[j] * TILE:(bcol[j] + 1) * TILE] = d[j]
        xq = from_bf16(to_bf16(np.asarray(x, dtype=np.float32))).reshape(self.batch, self.n_pre)
        return (wq[:self.n_post, :self.n_pre] @ xq.T).T

    def close(self):
        self.nat.close()
