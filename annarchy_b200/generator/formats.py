"""Storage formats of rate-coded projections and their conversion from CSR.

Containers restated from the reference's headers (ANNarchy/include/*.hpp):

* ELL   (ELLMatrix.hpp:76, init :290-363): rows padded to the longest row,
        column-major slots (slot k of row r at k*rows + r), empty slots hold
        -1 (the reference uses the index type's maximum).
* ELL-R (ELLRMatrix.hpp:73, init :245): ELL plus the length of every row.
* SELL  (SELLMatrix.hpp:69, init :285): slices of C rows, each padded to its
        own longest row; the reference uses C = 32 rows and keeps the row
        order. This backend also sorts rows by length inside windows of
        sigma rows (SELL-C-sigma) and keeps the permutation.
* BSR   (BSRMatrix.hpp:41, init :149-260): dense t x t tiles, block-row
        pointer and block-column indices, column-major tiles.
* HYB   (HYBMatrix.hpp:68, init :279): an ELL part of width k plus a COO
        tail holding the rest of every longer row; the reference picks k as
        the modal row length (HYBMatrix.hpp:84-104).

In double precision every format sums each row in ascending pre rank, so
its result equals CSR bit for bit, except HYB, which adds the ELL part and
then the tail of a row (the reference's HYB differs from CSR the same way).

This backend adds one schedule of its own, without a counterpart among the
reference's containers:

* PCSR  (panelled CSR, single precision only): the pre-synaptic columns cut
        into panels that fit in one CTA's shared memory, one CSR per panel
        with 16-bit column indices, and a table assigning each CTA a row
        range of one panel with about the same number of synapses. In double
        precision a PCSR projection is summed as CSR (ascending pre rank).
"""
from __future__ import annotations

import numpy as np

RATE_FORMATS = ("csr", "ell", "ellr", "sell", "bsr", "hyb", "pcsr")


def csr_group(mean_row: float) -> int:
    """Lanes per row of the vector CSR kernel."""
    for g in (2, 4, 8, 16):
        if mean_row <= 2 * g:
            return g
    return 32


def csr_bins(row_ptr, heavy_min: int = 0):
    """Rows split by length: (light rows, heavy rows) with heavy rows longer
    than max(1024, 16 x the mean); heavy rows get a CTA each."""
    rl = _lengths(row_ptr)
    if rl.size == 0:
        return np.zeros(0, np.int32), np.zeros(0, np.int32)
    cut = heavy_min or max(1024, int(16 * rl.mean()))
    heavy = np.nonzero(rl > cut)[0].astype(np.int32)
    light = np.nonzero(rl <= cut)[0].astype(np.int32)
    return light, heavy


def vec_group(mean_row: float) -> int:
    """Lanes per row of the vector-load CSR kernel (each lane takes 4
    entries per iteration)."""
    for g in (2, 4, 8, 16):
        if mean_row <= 8 * g:
            return g
    return 32


def _lengths(row_ptr):
    return np.diff(np.asarray(row_ptr, dtype=np.int64))


def ell_arrays(row_ptr, cols, w, width=None):
    """(cols, w, rl) column-major with `width` slots per row (default: max)."""
    rl = _lengths(row_ptr)
    rows = rl.size
    width = int(rl.max()) if width is None and rows else int(width or 0)
    ec = np.full((width, rows), -1, dtype=np.int32)
    ew = np.zeros((width, rows), dtype=np.float64)
    r_of = np.repeat(np.arange(rows), rl)
    k_of = np.arange(cols.size) - np.repeat(np.asarray(row_ptr[:-1], dtype=np.int64), rl)
    keep = k_of < width
    ec[k_of[keep], r_of[keep]] = cols[keep]
    ew[k_of[keep], r_of[keep]] = w[keep]
    return ec.ravel(), ew.ravel(), np.minimum(rl, width).astype(np.int32), width


def sell_arrays(row_ptr, cols, w, C=32, sigma=1):
    """SELL-C-sigma. Returns dict with slice_ptr, slice_len, cols, w, row_len
    (in sorted order) and perm (sorted position -> original row)."""
    rl = _lengths(row_ptr)
    rows = rl.size
    perm = np.arange(rows)
    if sigma > 1:
        for s0 in range(0, rows, sigma):
            s1 = min(rows, s0 + sigma)
            perm[s0:s1] = s0 + np.argsort(-rl[s0:s1], kind="stable")
    nsl = (rows + C - 1) // C
    slice_len = np.zeros(nsl, dtype=np.int32)
    rl_sorted = rl[perm]
    for s in range(nsl):
        seg = rl_sorted[s * C:(s + 1) * C]
        slice_len[s] = seg.max() if seg.size else 0
    slice_ptr = np.zeros(nsl + 1, dtype=np.int64)
    np.cumsum(slice_len.astype(np.int64) * C, out=slice_ptr[1:])
    sc = np.zeros(int(slice_ptr[-1]), dtype=np.int32)
    sw = np.zeros(int(slice_ptr[-1]), dtype=np.float64)
    starts = np.asarray(row_ptr[:-1], dtype=np.int64)
    pos = np.repeat(np.arange(rows, dtype=np.int64), rl_sorted)          # sorted position
    first = np.zeros(rows + 1, dtype=np.int64)
    np.cumsum(rl_sorted, out=first[1:])
    k = np.arange(pos.size, dtype=np.int64) - np.repeat(first[:-1], rl_sorted)
    slot = slice_ptr[pos // C] + k * C + pos % C
    src = np.repeat(starts[perm], rl_sorted) + k
    sc[slot] = cols[src]
    sw[slot] = w[src]
    return dict(slice_ptr=slice_ptr[:-1].astype(np.int32), slice_len=slice_len, cols=sc, w=sw,
                row_len=rl_sorted.astype(np.int32), perm=perm.astype(np.int32), nslices=nsl)


def hyb_width(row_ptr) -> int:
    """ELL width of the HYB split: the modal row length (HYBMatrix.hpp:84-104)."""
    rl = _lengths(row_ptr)
    if rl.size == 0:
        return 0
    counts = np.bincount(rl)
    return int(np.argmax(counts))


PCSR_MAX_ROWS = 4096


def pcsr_arrays(row_ptr, cols, w, n_pre, panel_width=16384, ctas=296, max_rows=PCSR_MAX_ROWS):
    """Panelled CSR. Returns dict(row_ptr (n_panels x (rows+1), int32,
    absolute offsets), col (uint16, relative to the panel), w (float64,
    reordered), cta_tab ((n_cta, 4) int32: panel, first row, end row, first
    entry in crow), crow (uint16: for each aligned 8-synapse chunk
    overlapping a CTA's synapse range, the row of its first synapse in the
    range, relative to the CTA's first row), n_panels, panel_width).
    Synapse arrays are padded by 8 zero entries past a multiple of 8. Each
    panel gets CTAs in proportion to its synapses, and a CTA's rows are cut
    where the cumulative synapse count crosses the panel's per-CTA share
    (and after max_rows rows, at most 65535)."""
    row_ptr = np.asarray(row_ptr, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    n_rows = row_ptr.size - 1
    panel_width = int(max(32, min(panel_width, 65536)) // 32 * 32)
    max_rows = int(min(max_rows, 65535))
    n_panels = max(1, -(-int(n_pre) // panel_width))
    rows_of = np.repeat(np.arange(n_rows, dtype=np.int64), np.diff(row_ptr))
    panel = (cols // panel_width).astype(np.uint16)
    # CSR order is row-major with ascending columns: a stable sort by panel
    # gives panel, then row, then column
    order = np.argsort(panel, kind="stable")
    counts = np.bincount(panel.astype(np.int64) * n_rows + rows_of,
                         minlength=n_panels * n_rows).reshape(n_panels, n_rows)
    rp = np.zeros((n_panels, n_rows + 1), dtype=np.int64)
    flat = np.cumsum(counts.reshape(-1))
    starts = np.concatenate([[0], flat])            # start of (panel, row) segments
    for p_ in range(n_panels):
        rp[p_] = starts[p_ * n_rows: (p_ + 1) * n_rows + 1]
    nnz = cols.size
    pad = (-nnz) % 8 + 8
    col16 = np.zeros(nnz + pad, dtype=np.uint16)
    col16[:nnz] = (cols[order] - panel[order].astype(np.int64) * panel_width).astype(np.uint16)
    wv = np.zeros(nnz + pad, dtype=np.float64)
    wv[:nnz] = np.asarray(w, dtype=np.float64)[order]
    per_panel = counts.sum(axis=1)
    tab = []
    for p_ in range(n_panels):
        if per_panel[p_] == 0:
            continue
        share = max(1, int(round(ctas * per_panel[p_] / max(nnz, 1))))
        target = per_panel[p_] / share
        cum = np.cumsum(counts[p_])
        r0 = 0
        while r0 < n_rows:
            # next cut: where the panel's cumulative count reaches the next share
            done = cum[r0 - 1] if r0 else 0
            r1 = int(np.searchsorted(cum, done + target, side="left")) + 1
            r1 = max(r0 + 1, min(r1, r0 + max_rows, n_rows))
            if cum[r1 - 1] > done:
                tab.append((p_, r0, r1))
            r0 = r1
    # per CTA: the row (relative to its first row) of the first synapse of
    # each aligned 8-synapse chunk that overlaps its synapse range
    full, crow = [], []
    base = 0
    for p_, r0, r1 in tab:
        seg = rp[p_, r0:r1 + 1]
        beg, end = int(seg[0]), int(seg[-1])
        a0 = beg & ~7
        first = np.maximum(np.arange(a0, end, 8, dtype=np.int64), beg)
        crow.append((np.searchsorted(seg, first, side="right") - 1).astype(np.uint16))
        full.append((p_, r0, r1, base))
        base += first.size
    cta_tab = np.asarray(full, dtype=np.int64).reshape(-1, 4).astype(np.int32)
    crow = np.concatenate(crow) if crow else np.zeros(0, np.uint16)
    return {"row_ptr": rp.astype(np.int32).reshape(-1), "col": col16, "w": wv, "cta_tab": cta_tab,
            "crow": np.concatenate([crow, np.zeros(8, np.uint16)]),
            "n_panels": n_panels, "panel_width": panel_width}


def bsr_arrays(post_rank, row_ptr, cols, w, n_pre, tile):
    """Dense t x t tiles over (post rank, pre rank). Returns block-row
    pointers, block columns, tile values (row-major inside a tile), the post
    rank of every tile row and the padded sizes."""
    rl = _lengths(row_ptr)
    rows_of = np.repeat(np.asarray(post_rank, dtype=np.int64), rl)
    n_post = int(post_rank.max()) + 1 if post_rank.size else 0
    nbr = (n_post + tile - 1) // tile
    br, bc = rows_of // tile, np.asarray(cols, dtype=np.int64) // tile
    key = br * ((n_pre + tile - 1) // tile) + bc
    ukey, inv = np.unique(key, return_inverse=True)
    nblk = ukey.size
    ubr = ukey // ((n_pre + tile - 1) // tile)
    ubc = ukey % ((n_pre + tile - 1) // tile)
    vals = np.zeros((nblk, tile, tile), dtype=np.float64)       # column-major tiles
    vals[inv, np.asarray(cols) % tile, rows_of % tile] = w
    brp = np.zeros(nbr + 1, dtype=np.int32)
    np.cumsum(np.bincount(ubr, minlength=nbr), out=brp[1:])
    return dict(block_row_ptr=brp, block_col=ubc.astype(np.int32), values=vals.reshape(-1),
                n_block_rows=nbr, n_blocks=nblk, n_post_pad=nbr * tile)


def select_format(proj, compiled) -> str:
    """Format used for storage_format='auto'. Single precision: the learned
    selector (annarchy_b200.selector, trained on the simulator's own timings)
    picks the schedule and sets its parameter (SELL window, BSR tile) in the
    projection's layout. Otherwise, or without a trained model, the
    reference's rule for rate-coded projections on the GPU
    (ANNarchy/core/Projection.py:691-789): mean row length <= 128 -> SELL
    (ELL-R when plastic), else CSR."""
    sched = getattr(proj, "_schedule", None)
    if sched:
        return sched
    m = proj._csr
    if not compiled.exact and not proj.plastic and not compiled.net._config.get("no_selector"):
        from .. import selector
        model = selector.default_model()
        if model is not None:
            s = model.choose(m)
            if "sell_sigma" in s:
                proj._sell_sigma = s["sell_sigma"]
            if "bsr_tile" in s:
                proj._bsr_tile_size = s["bsr_tile"]
            return s["format"]
    mean = m.nnz / max(1, (np.diff(m.indptr) > 0).sum())
    if mean <= 128:
        return "ellr" if proj.plastic else "sell"
    return "csr"


def create_format_arrays(compiled, proj, fmt, post_rank, row_ptr, cols, w, lay):
    nat = compiled.native
    k = proj.id
    W = compiled._w
    if fmt in ("ell", "ellr"):
        ec, ew, rl, width = ell_arrays(row_ptr, cols, w)
        nat.create(f"proj{k}__ell_col", ec)
        nat.create(f"proj{k}__ell_w", W(ew))
        if fmt == "ellr":
            nat.create(f"proj{k}__rl", rl)
        lay["width"] = width
    elif fmt == "sell":
        C = 32
        sigma = int(getattr(proj, "_sell_sigma", 0) or proj.net._config.get("sell_sigma", 1024))
        sigma = 1 if compiled.exact else sigma
        d = sell_arrays(row_ptr, cols, w, C=C, sigma=sigma)
        nat.create(f"proj{k}__slice_ptr", d["slice_ptr"])
        nat.create(f"proj{k}__slice_len", d["slice_len"])
        nat.create(f"proj{k}__sell_col", d["cols"])
        nat.create(f"proj{k}__sell_w", W(d["w"]))
        nat.create(f"proj{k}__sell_rl", d["row_len"])
        nat.create(f"proj{k}__perm", d["perm"])
        lay["C"] = C
    elif fmt == "hyb":
        width = hyb_width(row_ptr)
        ec, ew, rl, _ = ell_arrays(row_ptr, cols, w, width=width)
        nat.create(f"proj{k}__ell_col", ec)
        nat.create(f"proj{k}__ell_w", W(ew))
        nat.create(f"proj{k}__rl", rl)
        lay["width"] = width
        lens = _lengths(row_ptr)
        tail_len = np.maximum(lens - width, 0)
        tail_rows = np.nonzero(tail_len)[0]
        starts = np.asarray(row_ptr[:-1], dtype=np.int64)
        idx = np.concatenate([np.arange(starts[r] + width, starts[r] + lens[r]) for r in tail_rows]) \
            if tail_rows.size else np.zeros(0, dtype=np.int64)
        lay["coo_nnz"] = int(idx.size)
        lay["coo_rows"] = int(tail_rows.size)
        if idx.size:
            trp = np.zeros(tail_rows.size + 1, dtype=np.int32)
            np.cumsum(tail_len[tail_rows], out=trp[1:])
            nat.create(f"proj{k}__coo_row_ptr", trp)
            nat.create(f"proj{k}__coo_post", post_rank[tail_rows].astype(np.int32))
            nat.create(f"proj{k}__coo_row", np.repeat(tail_rows, tail_len[tail_rows]).astype(np.int32))
            nat.create(f"proj{k}__coo_col", cols[idx].astype(np.int32))
            nat.create(f"proj{k}__coo_w", W(w[idx]) if not compiled.exact else w[idx])
            from .codegen import grid_for
            lay["tail_grid"] = grid_for(int(idx.size) if not compiled.exact else int(tail_rows.size))
    elif fmt == "bsr":
        tile = int(getattr(proj, "_bsr_tile_size", 0) or proj.net._config.get("bsr_tile", 16))
        d = bsr_arrays(post_rank, row_ptr, cols, w, proj.pre_pop.size, tile)
        nat.create(f"proj{k}__bsr_row_ptr", d["block_row_ptr"])
        nat.create(f"proj{k}__bsr_col", d["block_col"])
        nat.create(f"proj{k}__bsr_val", W(d["values"]))
        lay.update(tile=tile, block_rows=d["n_block_rows"], n_post_pad=d["n_post_pad"])
    elif fmt == "pcsr":
        if compiled.exact:          # summed as CSR in double precision
            return
        cfg = proj.net._config
        pw = int(cfg.get("pcsr_panel", 16384))
        mr = int(cfg.get("pcsr_rows", PCSR_MAX_ROWS))
        sms = int(cfg.get("sm_count", 148))
        d = pcsr_arrays(row_ptr, cols, w, proj.pre_pop.size, panel_width=pw,
                        ctas=int(cfg.get("pcsr_ctas", 2 * sms)), max_rows=mr)
        nat.create(f"proj{k}__pc_row_ptr", d["row_ptr"])
        nat.create(f"proj{k}__pc_col", d["col"])
        nat.create(f"proj{k}__pc_w", W(d["w"]))
        nat.create(f"proj{k}__pc_cta", d["cta_tab"].reshape(-1))
        nat.create(f"proj{k}__pc_crow", d["crow"])
        block = int(cfg.get("pcsr_block", 1024))
        smem = 4 * d["panel_width"] + 8 * mr + 4
        resident = max(1, min(2048 // block, (228 * 1024) // (smem + 1024)))
        lay.update(n_panels=d["n_panels"], panel_width=d["panel_width"],
                   pc_ctas=int(d["cta_tab"].shape[0]), pc_max_rows=mr, pc_block=block,
                   pc_resident=resident)
    else:
        raise ValueError(f"unknown format {fmt!r}")


def refresh_format_weights(compiled, proj, w_flat):
    post_rank, row_ptr, cols, _ = proj.csr_population_ranks()
    lay = compiled.layout[proj.id]
    create_format_arrays(compiled, proj, lay["format"], post_rank, row_ptr, cols,
                         np.asarray(w_flat, dtype=np.float64), dict(lay))
