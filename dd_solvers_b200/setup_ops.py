"""Setup-time data preparation (runs once per operator, outside the solve loop).

Counterparts in the reference: ``SchwarzOperator.setup`` and its numba kernels
(``src/dd_solvers/dd_solvers/solvers.py:571-771``, dense block extraction
407-423, coarse matrix 426-481), ``Inv.setup`` (350-353) and ``csr_to_bsr``
(``src/dd_solvers/cpp/cusparse.cpp:22-107``). These are written with torch
tensor ops so they run on the GPU for large problems and on CPU tensors in
the host-side tests; no kernel of the solve path is involved.

HBM layouts produced here (all consumed by ``libddx.so``):

* SELL-32 matrix: ``slice_ptr`` (int64, nslices+1), ``slice_width`` (int32),
  ``cols`` (int32), ``vals`` (float64); entry ``j`` of row ``32 s + l`` at
  ``slice_ptr[s] + 32 j + l``; padding has value 0 and the row's own column.
* Inverse blocks: one flat buffer per precision; block ``i`` column-major with
  leading dimension ``ld_i = round_up(k_i, 16 / elem_size)`` at element offset
  ``blk_off[i]`` (16-byte aligned), rows ``k_i..ld_i-1`` zero; FP32 per-block
  power-of-two scales for low-precision storage.
* Transpose map: ``dof_ptr`` (int32, n+1), ``dof_src`` (int32): the positions of
  DOF ``d`` in the subdomain-major concatenation ``sub_idx`` in ascending order.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sps
import torch

ELEM_BYTES = {torch.float64: 8, torch.float32: 4, torch.bfloat16: 2, torch.float16: 2}
# |Q| <= 2**TARGET_EXP after scaling (FP16 uses its range: largest power of two
# below its maximum 65504 is 2**15; 2**14 keeps a factor-2 margin).
TARGET_EXP = {torch.float64: None, torch.float32: 0, torch.bfloat16: 0, torch.float16: 14}


# ---------------------------------------------------------------------------
# SELL-32
# ---------------------------------------------------------------------------

def csr_to_sell32(crow: torch.Tensor, col: torch.Tensor, val: torch.Tensor, return_positions: bool = False):
    """CSR -> SELL-32 (slice height 32, no row sorting).

    With ``return_positions`` also returns the SELL position of every CSR
    entry, so new values on the same pattern can be scattered in place.
    """
    dev = crow.device
    n = crow.numel() - 1
    nsl = (n + 31) // 32
    lens = (crow[1:] - crow[:-1]).to(torch.int64)
    lens_p = torch.zeros(nsl * 32, dtype=torch.int64, device=dev)
    lens_p[:n] = lens
    width = lens_p.view(nsl, 32).amax(dim=1)
    slice_ptr = torch.zeros(nsl + 1, dtype=torch.int64, device=dev)
    slice_ptr[1:] = torch.cumsum(width * 32, 0)
    total = int(slice_ptr[-1])
    rows_all = torch.arange(nsl * 32, device=dev)
    # padding default: own row (clamped to a valid column), value 0
    cols_s = torch.empty(total, dtype=torch.int32, device=dev)
    vals_s = torch.zeros(total, dtype=torch.float64, device=dev)
    # fill default columns slice by slice: position slice_ptr[s] + 32 j + l -> row 32 s + l
    pos = torch.arange(total, device=dev)
    sl = torch.searchsorted(slice_ptr, pos, right=True) - 1
    lrow = (pos - slice_ptr[sl]) % 32
    cols_s[:] = torch.clamp(sl * 32 + lrow, max=max(n - 1, 0)).to(torch.int32)
    # scatter real entries
    row_of = torch.repeat_interleave(torch.arange(n, device=dev), lens)
    j_in_row = torch.arange(int(crow[-1]), device=dev) - crow[:-1].to(torch.int64)[row_of]
    dst = slice_ptr[row_of // 32] + j_in_row * 32 + (row_of % 32)
    cols_s[dst] = col.to(torch.int32)
    vals_s[dst] = val.to(torch.float64)
    del rows_all
    if return_positions:
        return slice_ptr, width.to(torch.int32), cols_s, vals_s, dst
    return slice_ptr, width.to(torch.int32), cols_s, vals_s


# ---------------------------------------------------------------------------
# Subdomain maps
# ---------------------------------------------------------------------------

def transpose_map(sub_idx: torch.Tensor, n: int):
    """DOF -> positions in the subdomain-major list, ascending (stable sort)."""
    order = torch.argsort(sub_idx.to(torch.int64), stable=True)
    counts = torch.bincount(sub_idx.to(torch.int64), minlength=n)
    dof_ptr = torch.zeros(n + 1, dtype=torch.int64, device=sub_idx.device)
    dof_ptr[1:] = torch.cumsum(counts, 0)
    return dof_ptr.to(torch.int32), order.to(torch.int32)


RESTRICT_MAX_SLOTS = 16  # coarse rows one subdomain may touch (ddx_schwarz_restrict_sub)


def subdomain_restriction(ar_ptr, ar_col, ar_val, n_c: int, n: int, sub_ptr, sub_idx, slices: int = 1) -> dict:
    """Per-subdomain form of the hybrid restriction ``A_R y = sum_i (A_R R_i^T) y_i``
    (``ddx_schwarz_restrict_sub``), built with torch on the tensors' device.

    The coarse rows c with ``A_R[c, idx_i] != 0`` are subdomain i's slots
    (ascending c); pair ``q = slot_base[i] + slot`` (pairs ascending in (i, c)).
    Position p of the subdomain-major list carries its entries (slot,
    ``A_R[c, sub_idx[p]]``) in ascending c: the first two as
    ``f_slot[2p + e]`` (uint8, 255 for none) and ``f_val[2p + e]``, the others
    in ``ov_ptr[p] .. ov_ptr[p+1]`` of ``ov_slot`` / ``ov_val``. ``sum_ptr`` / ``sum_pair`` list, per coarse
    row, its pairs in ascending subdomain order. With ``slices`` > 1 (a local
    apply that splits each block into parts, part s writing ylocal slice s at
    row offset s * sum k_i) the positions of every slice carry the same
    entries (the per-position arrays cover ``slices * sum k_i`` rows).

    ``max_slots`` is the largest slot count; the kernel takes at most
    ``RESTRICT_MAX_SLOTS``.
    """
    dev = ar_ptr.device
    ptr = ar_ptr.to(torch.int64)
    col = ar_col.to(torch.int64)
    val = ar_val.to(torch.float64)
    # A_R^T by DOF: the coarse rows c (ascending) and values of column d of A_R
    rows = torch.repeat_interleave(torch.arange(n_c, device=dev), ptr[1:] - ptr[:-1])
    order = torch.argsort(col * n_c + rows)
    t_c, t_v = rows[order], val[order]
    t_ptr = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    t_ptr[1:] = torch.cumsum(torch.bincount(col, minlength=n), 0)
    sp = sub_ptr.to(dev, torch.int64)
    d = sub_idx.to(dev, torch.int64)
    n_sub = int(sp.numel()) - 1
    total = int(d.numel())
    sub = torch.repeat_interleave(torch.arange(n_sub, device=dev), sp[1:] - sp[:-1])
    cnt = t_ptr[d + 1] - t_ptr[d]
    n_e = int(cnt.sum())
    first = torch.cumsum(cnt, 0) - cnt
    e_pos = torch.repeat_interleave(torch.arange(total, device=dev), cnt)
    src = torch.repeat_interleave(t_ptr[d] - first, cnt) + torch.arange(n_e, device=dev)
    e_c = t_c[src]
    e_val = t_v[src]
    pkey = sub[e_pos] * n_c + e_c
    pairs, inv = torch.unique(pkey, sorted=True, return_inverse=True)
    n_pairs = int(pairs.numel())
    p_sub, p_c = pairs // n_c, pairs % n_c
    n_slots = torch.bincount(p_sub, minlength=n_sub)
    slot_base = torch.cumsum(n_slots, 0) - n_slots
    e_slot = inv - slot_base[sub[e_pos]]
    # the first two entries of every position, stored directly (entries are
    # grouped by position, c ascending); the rest in the overflow lists
    f_slot = torch.full((total, 2), 255, dtype=torch.int64, device=dev)
    f_val = torch.zeros(total, 2, dtype=torch.float64, device=dev)
    rank = torch.arange(n_e, device=dev) - first[e_pos]  # entry's index within its position
    direct = rank < 2
    f_slot[e_pos[direct], rank[direct]] = e_slot[direct]
    f_val[e_pos[direct], rank[direct]] = e_val[direct]
    ov_slot, ov_val = e_slot[~direct], e_val[~direct]
    ov_cnt = (cnt - 2).clamp(min=0)
    f_slot, f_val = f_slot.reshape(-1), f_val.reshape(-1)
    S = max(int(slices), 1)
    if S > 1:
        f_slot, f_val, ov_cnt = f_slot.repeat(S), f_val.repeat(S), ov_cnt.repeat(S)
        ov_slot, ov_val = ov_slot.repeat(S), ov_val.repeat(S)
    ov_ptr = torch.zeros(S * total + 1, dtype=torch.int64, device=dev)
    ov_ptr[1:] = torch.cumsum(ov_cnt, 0)
    # each coarse row's pairs in ascending subdomain order
    o2 = torch.argsort(p_c * max(n_sub, 1) + p_sub)
    sum_ptr = torch.zeros(n_c + 1, dtype=torch.int64, device=dev)
    sum_ptr[1:] = torch.cumsum(torch.bincount(p_c, minlength=n_c), 0)
    max_slots = int(n_slots.max()) if n_sub else 0
    assert int(ov_ptr[-1]) < 2 ** 31, "restriction plan too large for 32-bit entry offsets"
    u8 = lambda t: t.clamp(max=255).to(torch.uint8).contiguous()  # noqa: E731 (slots >= 255 are refused by max_slots)
    return {"n_pairs": n_pairs, "max_slots": max_slots, "slot_base": slot_base.to(torch.int32),
            "n_slots": n_slots.to(torch.int32), "f_slot": u8(f_slot), "f_val": f_val.contiguous(),
            "ov_ptr": ov_ptr.to(torch.int32), "ov_slot": u8(ov_slot), "ov_val": ov_val.contiguous(),
            "sum_ptr": sum_ptr.to(torch.int32), "sum_pair": o2.to(torch.int32), "slices": S}


def extract_blocks(crow, col, val, sub_ptr, sub_idx, first: int, last: int, kpad: int) -> torch.Tensor:
    """Dense local matrices ``A[idx_i][:, idx_i]`` for subdomains ``first..last-1``.

    Returns ``(last-first, kpad, kpad)`` FP64 with the identity in the padding
    rows/columns (so every block stays invertible). Entries are located with a
    sorted-key search, the vectorised form of the reference's per-row scan
    (``solvers.py:407-423``); a subdomain's indices may come in any order (a
    sharded rank numbers its owned DOFs before its ghosts).
    """
    dev = crow.device
    n = crow.numel() - 1
    p0, p1 = int(sub_ptr[first]), int(sub_ptr[last])
    B = last - first
    out = torch.zeros(B, kpad, kpad, dtype=torch.float64, device=dev)
    ks = (sub_ptr[first + 1:last + 1] - sub_ptr[first:last]).to(torch.int64)
    # identity padding
    ar = torch.arange(kpad, device=dev)
    pad = ar[None, :] >= ks[:, None]
    out.diagonal(dim1=1, dim2=2)[pad] = 1.0
    if p1 == p0:
        return out
    pos = torch.arange(p0, p1, device=dev)
    s_loc = torch.repeat_interleave(torch.arange(B, device=dev), ks)
    lrow = pos - sub_ptr[first:last].to(torch.int64)[s_loc]
    g = sub_idx[p0:p1].to(torch.int64)
    mkey = s_loc * n + g
    order = torch.argsort(mkey, stable=True)  # the identity for ascending index lists
    mkey = mkey[order]
    rs = crow[g].to(torch.int64)
    cnt = crow[g + 1].to(torch.int64) - rs
    e_row = torch.repeat_interleave(torch.arange(p1 - p0, device=dev), cnt)
    e_off = torch.arange(int(cnt.sum()), device=dev) - torch.repeat_interleave(torch.cumsum(cnt, 0) - cnt, cnt)
    e_idx = rs[e_row] + e_off
    ecol = col[e_idx].to(torch.int64)
    key = s_loc[e_row] * n + ecol
    hit = torch.searchsorted(mkey, key)
    hit_c = torch.clamp(hit, max=mkey.numel() - 1)
    ok = mkey[hit_c] == key
    lcol = order[hit_c] - (sub_ptr[first:last].to(torch.int64)[s_loc[e_row]] - p0)
    out[s_loc[e_row][ok], lrow[e_row][ok], lcol[ok]] = val[e_idx][ok].to(torch.float64)
    return out


def block_scales(inv: torch.Tensor, dtype: torch.dtype) -> torch.Tensor:
    """Per-block power-of-two scales (FP32) for low-precision storage."""
    t = TARGET_EXP[dtype]
    B = inv.shape[0]
    if t is None:
        return torch.ones(B, dtype=torch.float32, device=inv.device)
    amax = inv.abs().reshape(B, -1).amax(dim=1)
    amax = torch.where(amax > 0, amax, torch.ones_like(amax))
    m, e = torch.frexp(amax)  # amax = m * 2**e, m in [0.5, 1)
    e = torch.where(m == 0.5, e - 1, e)  # exact powers of two
    return torch.ldexp(torch.ones_like(amax), (e - t).to(torch.int32)).to(torch.float32)


def quantize(inv: torch.Tensor, scales: torch.Tensor, dtype: torch.dtype) -> torch.Tensor:
    """``Q = (B / s)`` rounded FP64 -> FP32 -> dtype (round to nearest even)."""
    q = inv / scales.to(torch.float64)[:, None, None]
    if dtype == torch.float64:
        return q
    return q.to(torch.float32).to(dtype)


SYM_T = 32  # edge of the symmetric-layout tiles


def sym_chunk_swizzle(r: torch.Tensor, elem_bytes: int) -> torch.Tensor:
    """XOR applied to the 16-byte chunk index of tile row ``r`` in the
    symmetric layout, so that eight consecutive rows read at the same chunk
    hit eight different 16-byte bank groups (rows of 64 B for 16-bit types:
    ``(r >> 1) & 3``; rows of 128/256 B for FP32/FP64: ``r & 7``)."""
    return ((r >> 1) & 3) if elem_bytes == 2 else (r & 7)


def sym_tile_index(elem_bytes: int, device) -> torch.Tensor:
    """Storage position of element (r, c) of a 32 x 32 tile: row-major rows of
    32 elements, 16-byte chunk ``c // V`` of row r stored at chunk
    ``(c // V) ^ sym_chunk_swizzle(r)`` (V = 16 / elem_bytes elements)."""
    V = 16 // elem_bytes
    r = torch.arange(SYM_T, device=device)[:, None]
    c = torch.arange(SYM_T, device=device)[None, :]
    return (r * SYM_T + ((c // V) ^ sym_chunk_swizzle(r, elem_bytes)) * V + (c % V)).reshape(-1)


class BlockStore:
    """Inverse blocks of one precision, quantised with a per-block power-of-two scale.

    ``layout="sym"`` (the default of the Schwarz operators): the FP64 inverse
    is symmetrised, ``(B + B^T) / 2``, before rounding, so the stored ``Q`` is
    exactly symmetric and only its upper-triangle 32 x 32 tiles are kept:
    block i (k rows, ``nt = ceil(k / 32)``) holds the ``nt (nt + 1) / 2`` tiles
    ``(I, J), I <= J`` in row-major order of (I, J), each 1024 elements in the
    swizzled row-major layout of ``sym_tile_index``, zero beyond k, starting at
    element ``blk_off[i]`` (16-byte aligned). About half the bytes of the full
    block. ``layout="colmajor"``: the full block column-major with leading
    dimension ``round_up(k, 16 B / element)``.
    """

    def __init__(self, ks: np.ndarray, dtype: torch.dtype, device, layout: str = "colmajor"):
        assert layout in ("colmajor", "sym")
        self.dtype = dtype
        self.layout = layout
        self.V = 16 // ELEM_BYTES[dtype]
        self.ks = ks.astype(np.int64)
        self.lds = ((self.ks + self.V - 1) // self.V) * self.V
        if layout == "sym":
            nt = (self.ks + SYM_T - 1) // SYM_T
            sizes = nt * (nt + 1) // 2 * (SYM_T * SYM_T)
        else:
            sizes = self.ks * self.lds
        off = np.zeros(len(ks) + 1, dtype=np.int64)
        np.cumsum(sizes, out=off[1:])
        self.off_np = off
        self.total = int(off[-1])
        self.data = torch.zeros(max(self.total, self.V), dtype=dtype, device=device)
        self.blk_off = torch.as_tensor(off[:-1], device=device)
        self.scale = torch.ones(len(ks), dtype=torch.float32, device=device)
        self._sw = sym_tile_index(ELEM_BYTES[dtype], device) if layout == "sym" else None
        # 16-bit symmetric blocks whose rounding made them indefinite are
        # re-rounded with a diagonal shift (see _guard_spd); {block: shift}
        self.spd_guard = True
        self.shifted: dict[int, float] = {}

    @property
    def nbytes(self) -> int:
        return self.total * ELEM_BYTES[self.dtype]

    def put(self, first: int, inv: torch.Tensor) -> None:
        """Stores blocks ``first..first+B-1`` from a padded (B, kpad, kpad) FP64 batch."""
        B = inv.shape[0]
        if self.layout == "sym":
            inv = 0.5 * (inv + inv.transpose(1, 2))
        sc = block_scales(inv, self.dtype)
        q = quantize(inv, sc, self.dtype)
        if self.spd_guard and self.dtype in (torch.bfloat16, torch.float16) and self.layout == "sym":
            q, sc = self._guard_spd(first, inv, q, sc)
        self.scale[first:first + B] = sc
        if self.layout == "sym":
            for b in range(B):
                i = first + b
                k = int(self.ks[i])
                if k == 0:
                    continue
                nt = (k + SYM_T - 1) // SYM_T
                full = torch.zeros(nt * SYM_T, nt * SYM_T, dtype=self.dtype, device=q.device)
                full[:k, :k] = q[b, :k, :k]
                tiles = full.view(nt, SYM_T, nt, SYM_T).permute(0, 2, 1, 3)  # [I, J, r, c]
                I, J = torch.triu_indices(nt, nt, device=q.device)
                up = tiles[I, J].reshape(-1, SYM_T * SYM_T)
                sw = torch.empty_like(up)
                sw[:, self._sw] = up
                self.data[self.off_np[i]:self.off_np[i + 1]] = sw.reshape(-1)
            return
        qt = q.transpose(1, 2)  # column-major: row c of qt is column c of q
        ks_b = np.asarray(self.ks[first:first + B])
        for kk in np.unique(ks_b):
            kk = int(kk)
            if kk == 0:
                continue
            sel = np.nonzero(ks_b == kk)[0]
            if kk > 64:  # few large blocks: one slice copy each
                for b in sel:
                    i = first + int(b)
                    ld = int(self.lds[i])
                    dst = self.data[self.off_np[i]:self.off_np[i] + kk * ld].view(kk, ld)
                    dst[:, :kk] = qt[b, :kk, :kk]
                continue
            # many small blocks of one size: one scatter per group of <= 2^22 entries
            ld = int(self.lds[first + int(sel[0])])
            cr = (torch.arange(kk, device=q.device)[:, None] * ld
                  + torch.arange(kk, device=q.device)[None, :]).reshape(-1)  # column c, row r
            step = max(1, (1 << 22) // (kk * kk))
            for a in range(0, len(sel), step):
                part = sel[a:a + step]
                offs = torch.as_tensor(self.off_np[first + part], device=q.device)
                dst = (offs[:, None] + cr[None, :]).reshape(-1)
                src = qt[torch.as_tensor(part, device=q.device), :kk, :kk].reshape(-1)
                self.data[dst] = src

    def _guard_spd(self, first: int, inv: torch.Tensor, q: torch.Tensor, sc: torch.Tensor):
        """Keeps every rounded 16-bit block positive definite.

        The inverse of a very ill-conditioned local block (cond ~1e5-1e6, the
        lognormal-coefficient outliers among thousands of subdomains) has its
        smallest eigenvalues below the 16-bit rounding error of its entries:
        rounding can make it indefinite, and PCG with an indefinite
        preconditioner stalls. Each rounded block is tested with a Cholesky
        factorisation of its dequantised FP64 form. A block that fails gets
        ``sigma I`` added before rounding again, with the smallest sigma (from
        twice the gap between half the block's smallest exact eigenvalue lam
        and the rounded block's smallest eigenvalue, doubled as needed) whose
        rounded block has all eigenvalues above lam / 2: the shift moves only
        the few eigenvalues the rounding pushed below zero, and little more.
        Blocks that pass, and blocks that are not positive definite before
        rounding either, are unchanged.
        """
        B, kb = inv.shape[0], inv.shape[-1]
        ks = torch.as_tensor(self.ks[first:first + B], device=inv.device)
        pad = (torch.arange(kb, device=inv.device)[None, :] >= ks[:, None]).to(torch.float64)

        def deq(qb, sb):
            return qb.to(torch.float64) * sb.to(torch.float64)[..., None, None]

        def spd(D, padb):
            D.diagonal(dim1=-2, dim2=-1).add_(padb)  # D is a fresh dequantised copy
            return torch.linalg.cholesky_ex(D)[1] == 0

        ok = spd(deq(q, sc), pad)
        bad = torch.nonzero(~ok).flatten().tolist()
        dev = inv.device
        for b in bad:
            k = int(ks[b])
            Bk = inv[b, :k, :k]
            lam = float(torch.linalg.eigvalsh(Bk)[0])
            if not lam > 0.0:
                continue  # not positive definite before rounding either: nothing to keep
            lam_q = float(torch.linalg.eigvalsh(deq(q[b, :k, :k], sc[b]))[0])
            eye = torch.eye(k, dtype=torch.float64, device=dev)
            sigma = 2.0 * (0.5 * lam - lam_q)
            for _ in range(20):
                Bs = Bk + sigma * eye
                ss = block_scales(Bs[None], self.dtype)
                qs = quantize(Bs[None], ss, self.dtype)[0]
                if bool(spd(deq(qs, ss[0]) - 0.5 * lam * eye, torch.zeros(k, dtype=torch.float64, device=dev))):
                    break
                sigma *= 2.0
            else:
                raise RuntimeError(f"block {first + b}: no positive-definite {self.dtype} rounding found")
            q[b] = 0
            q[b, :k, :k] = qs
            sc[b] = ss[0]
            self.shifted[first + b] = sigma
        return q, sc

    def dense_q(self, i: int) -> torch.Tensor:
        """Stored (quantised, unscaled) block i as a dense [row, col] k x k tensor."""
        k = int(self.ks[i])
        if self.layout == "sym":
            nt = (k + SYM_T - 1) // SYM_T
            sw = self.data[self.off_np[i]:self.off_np[i + 1]].view(-1, SYM_T * SYM_T)
            up = sw[:, self._sw].view(-1, SYM_T, SYM_T)
            full = torch.zeros(nt, nt, SYM_T, SYM_T, dtype=self.dtype, device=self.data.device)
            I, J = torch.triu_indices(nt, nt, device=self.data.device)
            full[I, J] = up
            full[J, I] = up.transpose(1, 2)
            return full.permute(0, 2, 1, 3).reshape(nt * SYM_T, nt * SYM_T)[:k, :k]
        ld = int(self.lds[i])
        d = self.data[self.off_np[i]:self.off_np[i] + k * ld].view(k, ld)[:, :k]
        return d.transpose(0, 1)

    def block(self, i: int) -> torch.Tensor:
        """Dequantised FP64 block i (for tests and requantisation)."""
        return self.dense_q(i).to(torch.float64) * float(self.scale[i])


UMMA_M = 128  # rows per tensor-core tile
UMMA_K = 64   # 16-bit columns per tile (one 128-byte swizzle row)


def umma_tile_rows(k: int) -> list[int]:
    """Rows stored for each 128-row tile of a k x k block (multiples of 8)."""
    rows = []
    for m0 in range(0, k, UMMA_M):
        r = min(UMMA_M, k - m0)
        rows.append((r + 7) // 8 * 8)
    return rows


def swizzle128_index(device) -> torch.Tensor:
    """Position of element (r, c) of a (128, 64) 16-bit tile in the K-major
    128-byte-swizzled layout: row r at byte 128 r, 16-byte chunk c // 8 stored
    at chunk (c // 8) ^ (r % 8)."""
    r = torch.arange(UMMA_M, device=device)[:, None]
    c = torch.arange(UMMA_K, device=device)[None, :]
    return (r * UMMA_K + (((c // 8) ^ (r % 8)) * 8) + (c % 8)).reshape(-1)


class UmmaTileStore:
    """16-bit inverse blocks pre-arranged as tensor-core A tiles.

    Subdomain ``i`` (size ``k``) is cut into ``ceil(k/128)`` row tiles by
    ``ceil(k/64)`` column tiles, stored row-tile-major at byte offset
    ``tile_off[i]``. Tile ``(m, t)`` holds ``rows_m`` rows (``umma_tile_rows``)
    of 64 columns in the K-major 128-byte-swizzled shared-memory layout, so one
    contiguous bulk copy lands it ready for ``tcgen05.mma``. Columns ``>= k``
    and padding rows are zero. Built from a ``BlockStore`` of the same type
    (either layout), so both hold identical values.
    """

    def __init__(self, src: "BlockStore"):
        assert src.dtype in (torch.bfloat16, torch.float16)
        dev = src.data.device
        self.dtype = src.dtype
        ks = src.ks
        sizes = []
        for k in ks:
            k = int(k)
            nK = (k + UMMA_K - 1) // UMMA_K
            sizes.append(sum(umma_tile_rows(k)) * nK * UMMA_K)
        off = np.zeros(len(ks) + 1, dtype=np.int64)
        np.cumsum(np.asarray(sizes, dtype=np.int64), out=off[1:])
        self.off_np = off
        self.data = torch.zeros(max(int(off[-1]), 8), dtype=src.dtype, device=dev)
        self.tile_off = torch.as_tensor(off[:-1] * 2, device=dev)  # bytes
        self.scale = src.scale
        sw = swizzle128_index(dev)
        for i, k in enumerate(ks):
            k = int(k)
            if k == 0:
                continue
            nK = (k + UMMA_K - 1) // UMMA_K
            rows = umma_tile_rows(k)
            full = torch.zeros(len(rows) * UMMA_M, nK * UMMA_K, dtype=src.dtype, device=dev)
            full[:k, :k] = src.dense_q(i)  # [row, col]
            tiles = full.view(len(rows), UMMA_M, nK, UMMA_K).permute(0, 2, 1, 3).reshape(len(rows), nK, -1)
            sw_tiles = torch.empty_like(tiles)
            sw_tiles[:, :, sw] = tiles
            o = int(off[i])
            for m, rm in enumerate(rows):
                n_el = rm * UMMA_K
                seg = sw_tiles[m, :, :n_el].reshape(-1)
                self.data[o:o + seg.numel()] = seg
                o += seg.numel()

    @property
    def nbytes(self) -> int:
        return int(self.off_np[-1]) * 2


class UmmaSymTileStore:
    """16-bit symmetric inverse blocks as upper-triangle 128 x 128 tensor-core tiles.

    Subdomain ``i`` (size ``k``, ``nt = ceil(k/128)``) holds its tiles ``(I, J),
    I <= J`` in row-major order of (I, J) from byte ``tile_off[i]``; each tile
    is two 128 x 64 halves (tile columns 0-63, then 64-127) in the K-major
    128-byte-swizzled layout of ``UmmaTileStore``, zero beyond k: 32 KB per
    tile, one bulk copy per tile. The tensor-core kernel uses each tile for
    ``T X_J`` and ``T^T X_I``. Built from a ``BlockStore`` whose blocks are
    exactly symmetric (``layout="sym"``).
    """

    TILE = 128

    def __init__(self, src: "BlockStore"):
        assert src.dtype in (torch.bfloat16, torch.float16) and src.layout == "sym"
        dev = src.data.device
        T = self.TILE
        self.dtype = src.dtype
        ks = src.ks
        nt = (ks.astype(np.int64) + T - 1) // T
        sizes = nt * (nt + 1) // 2 * T * T
        off = np.zeros(len(ks) + 1, dtype=np.int64)
        np.cumsum(sizes, out=off[1:])
        self.off_np = off
        self.data = torch.zeros(max(int(off[-1]), 8), dtype=src.dtype, device=dev)
        self.tile_off = torch.as_tensor(off[:-1] * 2, device=dev)  # bytes
        self.scale = src.scale
        sw = swizzle128_index(dev)
        for i, k in enumerate(ks):
            k = int(k)
            if k == 0:
                continue
            n = int(nt[i])
            full = torch.zeros(n * T, n * T, dtype=src.dtype, device=dev)
            full[:k, :k] = src.dense_q(i)
            tiles = full.view(n, T, n, T).permute(0, 2, 1, 3)  # [I, J, r, c]
            I, J = torch.triu_indices(n, n, device=dev)
            up = tiles[I, J]  # (ntiles, 128, 128)
            halves = up.view(-1, T, 2, UMMA_K).permute(0, 2, 1, 3).reshape(-1, 2, T * UMMA_K)  # [tile, half, r*64+c]
            swz = torch.empty_like(halves)
            swz[:, :, sw] = halves
            self.data[off[i]:off[i + 1]] = swz.reshape(-1)

    @property
    def nbytes(self) -> int:
        return int(self.off_np[-1]) * 2


def invert_blocks(blocks: torch.Tensor, ks: torch.Tensor) -> torch.Tensor:
    """Inverse of each padded SPD block; padding rows/cols zeroed afterwards.

    Batched Cholesky factor and inverse (k^3 flops per block, half of LU's;
    1.7x faster than ``torch.linalg.inv`` at k = 2242 on B200); a batch with a
    block that is not numerically SPD falls back to the LU inverse.
    """
    L, info = torch.linalg.cholesky_ex(blocks)
    if bool((info != 0).any()):
        inv = torch.linalg.inv(blocks)
    else:
        inv = torch.cholesky_inverse(L)
        del L
    kpad = blocks.shape[-1]
    ar = torch.arange(kpad, device=blocks.device)
    keep = ar[None, :] < ks[:, None]
    mask = (keep[:, :, None] & keep[:, None, :]).to(inv.dtype)
    return inv * mask


def csr_torch(M: sps.csr_matrix, device) -> torch.Tensor:
    """SciPy CSR -> torch CSR on ``device`` (int64 indices, FP64 values)."""
    M = sps.csr_matrix(M)
    return torch.sparse_csr_tensor(torch.as_tensor(M.indptr.astype(np.int64), device=device),
                                   torch.as_tensor(M.indices.astype(np.int64), device=device),
                                   torch.as_tensor(M.data.astype(np.float64), device=device), M.shape)


def spgemm_sorted(X: torch.Tensor, Y: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """``X @ Y`` of two torch CSR matrices on the device (cuSPARSE SpGEMM through
    torch), returned as (crow, col, val) with the columns of every row sorted,
    so the stored order does not depend on the product routine."""
    Z = X @ Y
    crow = Z.crow_indices().to(torch.int64)
    col = Z.col_indices().to(torch.int64)
    val = Z.values().to(torch.float64)
    rows = torch.repeat_interleave(torch.arange(Z.shape[0], device=crow.device), crow[1:] - crow[:-1])
    order = torch.argsort(rows * Z.shape[1] + col)
    return crow, col[order], val[order]


def scipy_csr(A) -> sps.csr_matrix:
    if isinstance(A, sps.spmatrix) or isinstance(A, sps.sparray):
        return sps.csr_matrix(A)
    crow = A.crow_indices().cpu().numpy()
    col = A.col_indices().cpu().numpy()
    val = A.values().cpu().numpy().astype(np.float64)
    return sps.csr_matrix((val, col, crow), shape=tuple(A.shape))


def round_up(x: int, m: int) -> int:
    return (x + m - 1) // m * m


def batch_for(kpad: int, budget_bytes: int = 2 << 30) -> int:
    """Subdomains per setup batch so a padded FP64 batch (x3 for LU workspace)
    stays within the budget."""
    per = 3 * kpad * kpad * 8
    return max(1, budget_bytes // max(per, 1))


def ceil_log2(x: float) -> int:
    return int(math.ceil(math.log2(x)))
