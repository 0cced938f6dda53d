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

* PCSR  (panelled sliced ELL, single precision only): the pre-synaptic
        columns cut into panels that fit in one CTA's shared memory (16-bit
        column indices), the rows of each panel sorted by length and stored
        in 32-row column-major slices, each behind a header step naming its
        rows; CTAs and warps take equal step ranges (pcsr_arrays). In double
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


PCSR_HEADER = 0xF000       # column values from here on mark a slice's header step


def pcsr_arrays(row_ptr, cols, w, n_pre, post_rank=None, panel_width=16384, ctas=444,
                warps=16):
    """Panelled sliced ELL (the backend's single-precision schedule).

    The pre-synaptic columns are cut into panels of `panel_width` neurons
    (16-bit column indices relative to the panel, below PCSR_HEADER). Within
    a panel the rows that have synapses there are sorted by their count there
    (longest first) and cut into slices of 32 rows. A slice is stored as
    steps of 32 elements, one per row: a header step naming the rows, then
    element k of every row at step k + 1 (column 0 and weight 0 past a row's
    end). The header's entry for lane l holds v = post_rank[row] + 1 (0 for a
    padding lane): its column is PCSR_HEADER | (v >> 16), its weight slot
    the bits of v (32-bit weights) or of v & 0xffff (16-bit weights). The
    steps of all panels form one array. Every panel gets CTAs in proportion
    to its steps, every CTA an equal range of the panel's steps and every
    warp of it an equal part of that range, wherever slices begin or end.

    Returns dict(col uint16 and w float64 (32 per step; header weights 0),
    header (step indices of the headers), header_val (int64, 32 per header:
    v), cta_panel (int32 per CTA), warp_tab ((CTAs x warps, 3) int32: first
    step, end step, header step of the slice holding the first step),
    n_panels, panel_width, n_steps, padded (stored elements)).
    """
    row_ptr = np.asarray(row_ptr, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    w = np.asarray(w, dtype=np.float64)
    n_rows = row_ptr.size - 1
    post = np.arange(n_rows) if post_rank is None else np.asarray(post_rank, dtype=np.int64)
    panel_width = int(max(32, min(panel_width, PCSR_HEADER)) // 32 * 32)
    n_panels = max(1, -(-int(n_pre) // panel_width))
    rows_of = np.repeat(np.arange(n_rows, dtype=np.int64), np.diff(row_ptr))
    panel = cols // panel_width
    # (panel, row) segments in CSR order: a stable sort by panel keeps the
    # rows and their ascending columns
    order = np.argsort(panel, kind="stable")
    counts = np.bincount(panel[order] * n_rows + rows_of[order],
                         minlength=n_panels * n_rows).reshape(n_panels, n_rows)
    seg_start = np.concatenate([[0], np.cumsum(counts.reshape(-1))])
    col_sorted = cols[order] - panel[order] * panel_width
    w_sorted = w[order]
    col_parts, w_parts, val_parts, head_parts, panel_steps = [], [], [], [], []
    step0 = 0
    for p_ in range(n_panels):
        cnt = counts[p_]
        rows = np.nonzero(cnt)[0]
        if rows.size == 0:
            panel_steps.append(0)
            continue
        rows = rows[np.argsort(-cnt[rows], kind="stable")]          # longest first
        ns = -(-rows.size // 32)
        lane_rows = np.full(ns * 32, -1, dtype=np.int64)
        lane_rows[:rows.size] = rows
        lane_rows = lane_rows.reshape(ns, 32)
        lens = np.where(lane_rows >= 0, cnt[np.maximum(lane_rows, 0)], 0)   # (ns, 32)
        slen = lens.max(axis=1) + 1                                  # header + elements
        head = np.concatenate([[0], np.cumsum(slen)[:-1]])
        n = int(slen.sum())
        s_idx = np.repeat(np.arange(ns), slen)
        k_idx = np.arange(n) - np.repeat(head, slen) - 1             # -1 on headers
        valid = (k_idx[:, None] >= 0) & (k_idx[:, None] < lens[s_idx])
        src = seg_start[p_ * n_rows + np.maximum(lane_rows[s_idx], 0)] + k_idx[:, None]
        cpad = np.zeros((n, 32), dtype=np.int64)
        wpad = np.zeros((n, 32), dtype=np.float64)
        cpad[valid] = col_sorted[src[valid]]
        wpad[valid] = w_sorted[src[valid]]
        val = np.where(lane_rows >= 0, post[np.maximum(lane_rows, 0)] + 1, 0)   # (ns, 32)
        cpad[head] = PCSR_HEADER | (val >> 16)
        col_parts.append(cpad.reshape(-1))
        w_parts.append(wpad.reshape(-1))
        val_parts.append(val.reshape(-1))
        head_parts.append(step0 + head)
        panel_steps.append(n)
        step0 += n
    n_steps = step0
    cat = lambda parts, dt: (np.concatenate(parts) if parts else np.zeros(0)).astype(dt)
    col16 = cat(col_parts, np.uint16)
    wv = cat(w_parts, np.float64)
    header = cat(head_parts, np.int64)
    # CTAs: per panel in proportion to its steps; warps: equal parts of a CTA
    cta_panel, wtab = [], []
    base = 0
    for p_, n in enumerate(panel_steps):
        if n == 0:
            continue
        k = max(1, int(round(ctas * n / max(n_steps, 1))))
        edges = base + (n * np.arange(k + 1)) // k
        for a, b in zip(edges[:-1], edges[1:]):
            cta_panel.append(p_)
            we = a + ((b - a) * np.arange(warps + 1)) // warps
            wtab.append(np.stack([we[:-1], we[1:]], axis=1))
        base += n
    if not cta_panel:                                # no synapses: one idle CTA
        cta_panel = [0]
        wtab = [np.zeros((warps, 2), dtype=np.int64)]
    wtab = np.concatenate(wtab)
    at = np.maximum(np.searchsorted(header, wtab[:, 0], side="right") - 1, 0)
    first_head = header[at] if header.size else np.zeros_like(at)
    warp_tab = np.concatenate([wtab, first_head[:, None]], axis=1).astype(np.int32)
    return {"col": np.concatenate([col16, np.zeros(8, np.uint16)]),
            "w": np.concatenate([wv, np.zeros(8)]),
            "header": header, "header_val": cat(val_parts, np.int64),
            "cta_panel": np.asarray(cta_panel, dtype=np.int32), "warp_tab": warp_tab,
            "n_panels": n_panels, "panel_width": panel_width, "n_steps": int(n_steps),
            "padded": int(col16.size)}


def pcsr_weights(d, W):
    """The weight array of a pcsr layout in the device type (W converts
    float64 weights to float32 or to bfloat16 bits), headers filled in."""
    out = np.array(W(d["w"]))
    idx = (32 * d["header"][:, None] + np.arange(32)[None, :]).reshape(-1)
    v = d["header_val"]
    if out.dtype == np.uint16:
        out[idx] = (v & 0xFFFF).astype(np.uint16)
    else:
        out.view(np.uint32)[idx] = v.astype(np.uint32)
    return out


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
        sms = int(cfg.get("sm_count", 148))
        # two CTAs of 512 threads per SM (64 registers a thread: 10 steps per
        # chunk): on the 100k-neuron uniform, local and power-law matrices
        # 23.0 / 27.8 / 24.6 us against 23.7 / 34.3 / 28.7 us with three CTAs
        # of 384 threads (cold L2, float32 weights)
        block = int(cfg.get("pcsr_block", 512))
        pw = max(32, min(pw, PCSR_HEADER)) // 32 * 32
        resident = max(1, min(2048 // block, (228 * 1024) // (4 * pw + 1024 + 64), 2))
        resident = int(cfg.get("pcsr_resident", resident))
        # steps per chunk (two chunks in flight): what the launch's registers allow
        regs = 65536 // (block * resident) // 8 * 8
        unroll = int(cfg.get("pcsr_unroll", max(2, min(16, (regs - 14) // 5))))
        d = pcsr_arrays(row_ptr, cols, w, proj.pre_pop.size, post_rank=post_rank, panel_width=pw,
                        ctas=int(cfg.get("pcsr_ctas", resident * sms)), warps=block // 32)
        if d["padded"] >= 2 ** 31 - 64 or post_rank.size and int(np.max(post_rank)) >= 2 ** 28 - 2:
            raise ValueError(f"{proj.name}: too many synapses or neurons for the pcsr format")
        nat.create(f"proj{k}__pc_col", d["col"])
        nat.create(f"proj{k}__pc_w", pcsr_weights(d, W))
        nat.create(f"proj{k}__pc_cta", d["cta_panel"])
        nat.create(f"proj{k}__pc_warp", d["warp_tab"].reshape(-1))
        lay.update(n_panels=d["n_panels"], panel_width=d["panel_width"],
                   pc_ctas=int(d["cta_panel"].size), pc_block=block, pc_resident=resident,
                   pc_unroll=unroll)
    else:
        raise ValueError(f"unknown format {fmt!r}")


def refresh_format_weights(compiled, proj, w_flat):
    post_rank, row_ptr, cols, _ = proj.csr_population_ranks()
    lay = compiled.layout[proj.id]
    create_format_arrays(compiled, proj, lay["format"], post_rank, row_ptr, cols,
                         np.asarray(w_flat, dtype=np.float64), dict(lay))
