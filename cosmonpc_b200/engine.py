"""Device pipeline: meshes, spectra, shell fields and x-space contractions.

Every numeric step runs in libcosmonpc_b200.so kernels or cuFFT; torch only
allocates device memory and provides the stream.  Two precisions:

* ``"f64"`` -- the plain drop-in: float64 meshes, Z2D/D2Z transforms, FP64
  shell fields and FP64 contractions.
* ``"f32"`` -- the fast form: float32 meshes and shell fields (C2R/R2C),
  FP64 mode sums and FP64 accumulation of the x-space contractions.

Layout (see include/cosmonpc_b200.h): real meshes n^3 (z fastest), spectra
n x n x (n/2+1) complex (cuFFT R2C layout).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib, angular

PRECISION = {
    "f32": (_lib.F32, torch.float32, torch.complex64),
    "f64": (_lib.F64, torch.float64, torch.complex128),
}


def _device():
    if not torch.cuda.is_available():
        raise RuntimeError("cosmonpc_b200 needs a CUDA device; none is available")
    return torch.device("cuda", torch.cuda.current_device())


class PaintedMesh:
    """Unnormalised R2C spectra of one painted catalog (and its +1/2-cell twin).

    Stands in for the reference's painted ``RealField`` (mesh_generator.py:172-224):
    the interlaced combination is applied when an estimator finishes the forward
    transform, fused with its scaling and compensation.
    """

    def __init__(self, raw, n, boxsize, sampler, interlaced, n_gal, sum_w, precision):
        self.raw = raw
        self.n = n
        self.boxsize = float(boxsize)
        self.sampler = sampler
        self.window = _lib.WINDOW[sampler]
        self.interlaced = bool(interlaced)
        self.N_gal = n_gal
        self.sum_w = sum_w
        self.precision = precision
        self.used = False


def paint(pos, weight, n, boxsize, sampler, interlaced, precision="f64", sum_w=None):
    """Paint a catalog held on the device and return its forward spectra."""
    ctx = _lib.Context.get()
    code, rdt, cdt = PRECISION[precision]
    dev = _device()
    pos = pos.to(device=dev, dtype=torch.float64).contiguous()
    if weight is not None:
        weight = weight.to(device=dev, dtype=torch.float64).contiguous()
    nb = 2 if interlaced else 1
    mesh = torch.empty((nb, n, n, n), dtype=rdt, device=dev)
    ctx.paint(code, pos, weight, n, float(boxsize), _lib.WINDOW[sampler], mesh[0],
              mesh[1] if interlaced else None)
    spec = torch.empty((nb, n, n, n // 2 + 1), dtype=cdt, device=dev)
    ctx.r2c(code, n, nb, mesh, spec)
    del mesh
    if sum_w is None:
        sum_w = float(pos.shape[0]) if weight is None else float(weight.sum().item())
    return PaintedMesh(spec, n, boxsize, sampler, interlaced, int(pos.shape[0]), sum_w, precision)


def finish_delta(pm, scale, comp, k0, band=0.0):
    """Interlace-combine, scale and compensate in place; returns the spectrum view.

    A PaintedMesh is consumed by one estimator (as the reference's rfield is
    overwritten in place, clustering_estimator.py:808)."""
    if pm.used:
        raise ValueError("painted mesh already consumed by an estimator")
    pm.used = True
    ctx = _lib.Context.get()
    code = PRECISION[pm.precision][0]
    spec2 = pm.raw[1] if pm.interlaced else None
    ctx.forward_finish(code, pm.n, pm.boxsize, pm.raw[0], spec2, float(scale), comp, pm.window,
                       float(k0), band)
    return pm.raw[0]


def finish_delta_band(pm, scale, comp, k0, band_out_k):
    """finish_delta that also returns the finished spectrum zeroed at
    |k| >= band_out_k, written into the consumed +1/2-cell twin spectrum when
    the mesh is interlaced (a new buffer otherwise)."""
    if pm.used:
        raise ValueError("painted mesh already consumed by an estimator")
    pm.used = True
    ctx = _lib.Context.get()
    code = PRECISION[pm.precision][0]
    spec2 = pm.raw[1] if pm.interlaced else None
    out = spec2 if spec2 is not None else torch.empty_like(pm.raw[0])
    ctx.forward_finish_band(code, pm.n, pm.boxsize, pm.raw[0], spec2, float(scale), comp, pm.window,
                            float(k0), 0.0, out, float(band_out_k))
    return pm.raw[0], out


def kbin_counts(n, boxsize, edges):
    """Mode counts and sum |k| per bin (geometry only: kept per shape class
    while UNIT_SHELL_CACHE is on)."""
    key = None
    if UNIT_SHELL_CACHE:
        key = (int(n), float(boxsize), tuple(float(e) for e in edges), torch.cuda.current_device())
        hit = _kbin_cache.get(key)
        if hit is not None:
            torch.cuda.current_stream().wait_event(hit[2])  # written on another stream, maybe
            return hit[0], hit[1]
    ctx = _lib.Context.get()
    dev = _device()
    nb = len(edges) - 1
    counts = torch.empty(nb, dtype=torch.float64, device=dev)
    ksum = torch.empty(nb, dtype=torch.float64, device=dev)
    ctx.kbin_counts(n, float(boxsize), edges, counts, ksum)
    if key is not None:
        done = torch.cuda.Event()
        done.record()
        _kbin_cache[key] = (counts, ksum, done)
    return counts, ksum


# ------------------------------------------------------------ shell fields
# Extra elements between consecutive shell fields (0: contiguous batches,
# which cuFFT writes fastest).
FIELD_PAD = 0
# FP32 shell fields of n = 64/128/192/256 whose bins lie below k_Nyquist / 2 are
# synthesised and inverse-transformed by the fused band-limited kernels
# (cnpc_shell_fields) instead of shell spectra + cuFFT C2R.
FUSED_SHELLS = True


# FP32 Gram blocks on the tensor cores (cnpc_contract_gram_tc[_multi_g], TF32
# pairs, A operand in tensor memory) instead of the CUDA-core FFMA kernel.
# Off by default: at 256^3 with 40 x 20 outputs the tensor-core kernel takes
# 1.15-1.19 ms against 0.84 ms for the FFMA kernel (CUDA events).  Its time does
# not change with 20 rows instead of 40: the per-chunk hand-offs between its
# producer, converter and MMA warps (an mbarrier wait costs ~240 cycles even on
# a completed phase) bound it, not the copies or the MMAs.
GRAM_TC = False

# FP32 Gram blocks of several weight fields (the FFT S3 sums of several
# configurations) with the same columns share one launch
GRAM_MULTI = True

# diagonal data vectors contract only their same-bin component pairs
# (cnpc_contract_pairs) instead of whole Gram blocks
PAIR_LIST = True


def fused_shells_apply(n, boxsize, edges, bins, precision):
    if not FUSED_SHELLS or precision != "f32" or n not in (64, 128, 192, 256):
        return False
    kf = 2.0 * np.pi / float(boxsize)
    top = max(float(edges[b + 1]) for b in bins)
    return top / kf < n / 4.0


def leg_components(l, m):
    """Real component fields of the complex shell field of Y_lm (see header)."""
    if m == 0:
        return (0,) if l % 2 == 0 else (1,)
    return (0, 1)


class ShellFields:
    """Real shell fields c2r(src * Y_lm * mask_bin) synthesised in FFT batches.

    A leg is (l, m, source, conj) with source 0 (spectrum A), 1 (spectrum B) or
    2 (unit spectrum).  Fields are stored as rows of one [capacity, n^3] tensor.
    """

    def __init__(self, n, boxsize, edges, precision, spec_a, spec_b, capacity, fft_batch=None,
                 racah=True):
        self.n = n
        self.boxsize = float(boxsize)
        self.edges = np.asarray(edges, dtype=np.float64)
        self.precision = precision
        self.code, self.rdt, self.cdt = PRECISION[precision]
        self.spec_a = spec_a
        self.spec_b = spec_b
        self.racah = racah
        dev = _device()
        self.capacity = int(capacity)
        # rows padded off the 2^k-byte stride of an n^3 field (see FIELD_PAD)
        self.stride = n * n * n + FIELD_PAD
        self.fields = torch.empty((self.capacity, self.stride), dtype=self.rdt, device=dev)
        if fft_batch is None:  # the shape class's tuned batch depth
            from . import autotune

            fft_batch = autotune.fft_batch(n, boxsize, edges, precision)
        self.fft_batch = max(1, min(int(fft_batch), self.capacity))
        self._scratch = None
        self.slot = {}
        self.free = list(range(self.capacity))[::-1]
        self.persistent = False  # fields survive release calls (unit-shell cache)
        # cells the contractions run over: n^3, or the planes x <= n/2 while
        # pair_sums contracts parity-folded weights (fold_weights)
        self.ncell_contract = n * n * n
        self.ready = None        # event after the last synthesis (persistent fields)

    @property
    def scratch(self):
        """Half spectra of one FFT batch (only the cuFFT route needs them)."""
        if self._scratch is None:
            n = self.n
            self._scratch = torch.empty((self.fft_batch, n, n, n // 2 + 1), dtype=self.cdt, device=_device())
        return self._scratch

    def key(self, leg, b, comp):
        return (tuple(leg), int(b), int(comp))

    def release_all(self):
        if self.persistent:
            return
        self.slot.clear()
        self.free = list(range(self.capacity))[::-1]

    def release(self, keys):
        if self.persistent:
            return
        for k in keys:
            s = self.slot.pop(k, None)
            if s is not None:
                self.free.append(s)

    def ensure(self, keys):
        """Synthesise every (leg, bin, comp) in ``keys`` not yet resident."""
        ctx = _lib.Context.get()
        todo = [k for k in dict.fromkeys(keys) if k not in self.slot]
        if self.persistent and self.ready is not None:
            # fields another stream may still be writing
            torch.cuda.current_stream().wait_event(self.ready)
        if len(todo) > len(self.free) and self.persistent:
            # a persistent cache holding other shells: start over with this set,
            # once no stream still reads the old ones
            torch.cuda.synchronize()
            self.slot.clear()
            self.free = list(range(self.capacity))[::-1]
            todo = list(dict.fromkeys(keys))
        if len(todo) > len(self.free):
            raise MemoryError("shell-field cache too small for this block")
        harm_index = {}
        harmonics = []
        for i in range(0, len(todo), self.fft_batch):
            batch = todo[i:i + self.fft_batch]
            items = []
            for (leg, b, comp) in batch:
                l, m, src, conj = leg
                hk = (l, m)
                if hk not in harm_index:
                    harm_index[hk] = len(harmonics)
                    harmonics.append(angular.harmonic(l, m, self.racah))
                items.append(_lib.ShellItem(b, harm_index[hk], comp, src, 1 if conj else 0))
            if fused_shells_apply(self.n, self.boxsize, self.edges, [k[1] for k in batch], self.precision):
                slots = [self.free.pop() for _ in batch]
                ctx.shell_fields(self.n, self.boxsize, self.spec_a, self.spec_b, self.edges, harmonics, items,
                                 [self.fields[s] for s in slots])
                for k, s in zip(batch, slots):
                    self.slot[k] = s
                continue
            ctx.shell_spectra(self.code, self.n, self.boxsize, self.spec_a, self.spec_b, self.edges,
                              harmonics, items, self.scratch)
            slots = [self.free.pop() for _ in batch]
            # contiguous slots let one batched c2r write every field of the batch
            if slots == list(range(slots[0], slots[0] + len(slots))):
                ctx.c2r(self.code, self.n, len(batch), self.scratch, self.fields[slots[0]:slots[0] + len(slots)],
                        self.stride)
            else:
                for j, s in enumerate(slots):
                    ctx.c2r(self.code, self.n, 1, self.scratch[j], self.fields[s], self.stride)
            for k, s in zip(batch, slots):
                self.slot[k] = s
        if self.persistent and todo:
            self.ready = torch.cuda.Event()
            self.ready.record()


class HostCopy:
    """A device tensor copied to pinned host memory without blocking the host;
    ``get()`` waits only for that copy."""

    def __init__(self, t):
        self.host = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        self.host.copy_(t, non_blocking=True)
        self.event = None
        if not torch.cuda.is_current_stream_capturing():
            # inside a CUDA graph capture the copy becomes a graph node: whoever
            # replays the graph synchronises before reading
            self.event = torch.cuda.Event()
            self.event.record()

    def get(self):
        if self.event is not None:
            self.event.synchronize()
            return self.host.numpy()
        return self.host.numpy().copy()  # a graph's buffer is rewritten by its next replay


def _staged_rows(nr, nc, shared):
    pad = lambda x: (x + 7) // 8 * 8
    return 1 + pad(nr) + (0 if shared else pad(nc))


def contract(G, sf, rows, cols):
    """Device tensor T[i, j] = sum_x G F_rows[i] F_cols[j] (FP64), enqueued only.

    One Gram launch stages G plus the row and column fields of a chunk of
    cells; when the columns are a contiguous run of the rows they share the
    staged rows.  Blocks of rows x columns are split so a launch stages at most
    ~100 rows."""
    ctx = _lib.Context.get()
    ncell = sf.ncell_contract
    dev = _device()
    T = torch.zeros((len(rows), len(cols)), dtype=torch.float64, device=dev)
    if not rows or not cols:
        return T
    ridx = [sf.slot[k] for k in rows]
    cidx = [sf.slot[k] for k in cols]

    def shared(rr, cc):
        for off in range(0, len(rr) - len(cc) + 1):
            if rr[off:off + len(cc)] == cc:
                return True
        return False

    tc = sf.precision == "f32" and GRAM_TC
    if sf.precision == "f32":
        # one FP32 contraction launch covers at most 40 rows x 24 columns on the
        # tensor cores, 48 x 24 on the CUDA cores
        rb, cb = (40, 24) if tc else (48, 24)
        if len(ridx) <= rb and len(cidx) <= cb:
            blocks = [(0, len(ridx), 0, len(cidx))]
        else:
            blocks = [(r0, min(len(ridx), r0 + rb), c0, min(len(cidx), c0 + cb))
                      for r0 in range(0, len(ridx), rb) for c0 in range(0, len(cidx), cb)]
    elif len(ridx) <= 128 and len(cidx) <= 128 and _staged_rows(len(ridx), len(cidx), shared(ridx, cidx)) <= 100:
        blocks = [(0, len(ridx), 0, len(cidx))]
    else:
        blocks = [(r0, min(len(ridx), r0 + 48), c0, min(len(cidx), c0 + 48))
                  for r0 in range(0, len(ridx), 48) for c0 in range(0, len(cidx), 48)]
    for (r0, r1, c0, c1) in blocks:
        rr, cc = ridx[r0:r1], cidx[c0:c1]
        run = (lambda o: ctx.gram_tc(ncell, G, sf.fields, sf.stride, rr, cc, o)) if tc else \
            (lambda o: ctx.gram(sf.code, ncell, G, sf.fields, sf.stride, rr, cc, o))
        if (r1 - r0, c1 - c0) == (len(ridx), len(cidx)):
            run(T)
        else:
            out = torch.empty((len(rr), len(cc)), dtype=torch.float64, device=dev)
            run(out)
            T[r0:r1, c0:c1] = out
    return T


# ---------------------------------------------------- pair-sum assembly
class PairSpec:
    """One magnetic sub-configuration's sum_x G F1_i F2_j.

    mode "leg": F2 from its own leg; "eq": F2 = F1; "conj": F2 = sign * conj(F1).
    """

    def __init__(self, leg1, mode, leg2=None, sign=1.0):
        self.leg1 = tuple(leg1)
        self.mode = mode
        self.leg2 = tuple(leg2) if leg2 is not None else None
        self.sign = sign

    def row_keys(self, sf, bins):
        l, m = self.leg1[0], self.leg1[1]
        return [sf.key(self.leg1, b, c) for b in bins for c in leg_components(l, m)]

    def col_keys(self, sf, bins):
        leg = self.leg1 if self.mode != "leg" else self.leg2
        return [sf.key(leg, b, c) for b in bins for c in leg_components(leg[0], leg[1])]


def _assemble_entry(ps, t, bi, bj):
    """Complex S(bi, bj) of one pair spec from real component sums t(k1, k2)."""
    leg2 = ps.leg1 if ps.mode != "leg" else ps.leg2
    R1, I1 = (ps.leg1, bi, 0), (ps.leg1, bi, 1)
    R2, I2 = (leg2, bj, 0), (leg2, bj, 1)
    if ps.mode == "conj":
        re = t(R1, R2) + t(I1, I2)
        im = t(I1, R2) - t(R1, I2)
        return ps.sign * complex(re, im)
    re = t(R1, R2) - t(I1, I2)
    im = t(R1, I2) + t(I1, R2)
    return complex(re, im)


def _entry_keys(ps, sf, bi, bj):
    """The (row key, column key) component pairs _assemble_entry reads."""
    leg2 = ps.leg1 if ps.mode != "leg" else ps.leg2
    c1 = leg_components(ps.leg1[0], ps.leg1[1])
    c2 = leg_components(leg2[0], leg2[1])
    return [(sf.key(ps.leg1, bi, a), sf.key(leg2, bj, b)) for a in c1 for b in c2]


def assemble(ps, T, rows, cols, rbins, cbins):
    """Complex S[i, j] over the (rbins x cbins) block from the real Gram T
    (_assemble_entry for every entry, by index arrays; a component that is not
    a row or column of T reads as zero)."""
    nr, nc = len(rows), len(cols)
    ri = {k: i for i, k in enumerate(rows)}
    ci = {k: j for j, k in enumerate(cols)}
    Tx = np.zeros((nr + 1, nc + 1))
    Tx[:nr, :nc] = T
    leg2 = ps.leg1 if ps.mode != "leg" else ps.leg2
    r_re = [ri.get((ps.leg1, b, 0), nr) for b in rbins]
    r_im = [ri.get((ps.leg1, b, 1), nr) for b in rbins]
    c_re = [ci.get((leg2, b, 0), nc) for b in cbins]
    c_im = [ci.get((leg2, b, 1), nc) for b in cbins]
    rr = Tx[np.ix_(r_re, c_re)]
    ii = Tx[np.ix_(r_im, c_im)]
    ir = Tx[np.ix_(r_im, c_re)]
    ri_ = Tx[np.ix_(r_re, c_im)]
    if ps.mode == "conj":
        return ps.sign * ((rr + ii) + 1j * (ir - ri_))
    return (rr - ii) + 1j * (ri_ + ir)


def contract_pairs(G, sf, pairs):
    """Device tensor v[p] = sum_x G F_a F_b for the (key_a, key_b) pairs (FP64)."""
    ctx = _lib.Context.get()
    out = torch.empty(len(pairs), dtype=torch.float64, device=_device())
    for p0 in range(0, len(pairs), 256):
        chunk = pairs[p0:p0 + 256]
        ctx.contract_pairs(sf.code, sf.ncell_contract, G, sf.fields, sf.stride, [sf.slot[a] for a, _ in chunk],
                           [sf.slot[b] for _, b in chunk], out[p0:p0 + len(chunk)])
    return out


class DeferredPairSums:
    """Pair sums whose device Grams are still in flight; ``result()`` copies
    them to the host once and assembles the complex sums."""

    def __init__(self, pair_specs, k_bins, diagonal):
        self.pair_specs = pair_specs
        self.k_bins = k_bins
        self.diagonal = diagonal
        self.blocks = []
        # where the sums are computed: a NaN in them is checked against the
        # context's device status word (a bounded wait that gave up)
        self.ctx = _lib.Context.get()
        self.stream = None if torch.cuda.is_current_stream_capturing() else torch.cuda.current_stream()

    def _check_status(self, vals):
        if np.isnan(vals).any() and self.stream is not None:
            self.ctx.take_status(self.stream)  # raises DeviceTimeout after a timed-out wait

    def add(self, T, rows, cols, bi, bj):
        self.blocks.append((HostCopy(T), rows, cols, bi, bj))

    def add_pairs(self, vals, pairs, bins):
        self.blocks.append((HostCopy(vals), pairs, None, bins, None))

    def result(self):
        k_bins = self.k_bins
        results = [np.zeros((k_bins, k_bins) if not self.diagonal else k_bins, dtype=np.complex128)
                   for _ in self.pair_specs]
        for hc, rows, cols, bi, bj in self.blocks:
            if cols is None:  # pair-list sums of the diagonal
                vals = hc.get()
                self._check_status(vals)
                lookup = dict(zip(rows, vals))
                t = lambda k1, k2: lookup.get((k1, k2), 0.0)
                for r, ps in enumerate(self.pair_specs):
                    for b in bi:
                        results[r][b] = _assemble_entry(ps, t, b, b)
                continue
            T = hc.get()
            self._check_status(T)
            for r, ps in enumerate(self.pair_specs):
                S = assemble(ps, T, rows, cols, bi, bj)
                if self.diagonal:
                    results[r][bi] = np.diag(S)
                else:
                    results[r][bi[0]:bi[-1] + 1, bj[0]:bj[-1] + 1] = S
        return results


# FP32 sums over shells of the unit spectrum run over half the cells: the
# fields have the parity (-1)^l, so sum_x G F_a F_b is the sum over the planes
# x <= n/2 of the parity-folded weight (cnpc_field_parity_fold)
PARITY_FOLD = True


def fold_weights(groups, sf):
    """The groups' weights folded for sums over the planes x <= n/2, or None
    when the fold does not apply: FP32 shells of the unit spectrum only, and
    every pair of a group with the same parity (-1)^(l1 + l2)."""
    if not PARITY_FOLD or sf.precision != "f32" or sf.spec_a is not None or sf.spec_b is not None:
        return None
    ctx = _lib.Context.get()
    n = sf.n
    folded = []
    for (G, specs) in groups:
        signs = set()
        for ps in specs:
            leg2 = ps.leg1 if ps.mode != "leg" else ps.leg2
            if ps.leg1[2] != 2 or leg2[2] != 2:
                return None  # not unit-spectrum shells
            signs.add(-1 if (ps.leg1[0] + leg2[0]) % 2 else 1)
        if len(signs) != 1:
            return None
        out = torch.empty((n // 2 + 1) * n * n, dtype=G.dtype, device=G.device)
        ctx.field_parity_fold(sf.code, n, G, signs.pop(), out)
        folded.append((out, specs))
    return folded


def pair_sums(groups, sf, k_bins, diagonal, block_size):
    """Enqueue sum_x G F1 F2 for every group (G, [PairSpec, ...]) over all bins,
    with one shared shell-field cache; returns one DeferredPairSums per group
    (``result()`` gives complex arrays k_bins x k_bins, or k_bins in diagonal
    mode).

    Bins are processed in blocks of ``block_size`` rows x columns so that at most
    the fields of one row block and one column block are resident
    (clustering_estimator.py:911-981 bounds memory the same way).
    """
    folded = fold_weights(groups, sf)
    if folded is not None:
        sf.ncell_contract = (sf.n // 2 + 1) * sf.n * sf.n
        try:
            return _pair_sums(folded, sf, k_bins, diagonal, block_size)
        finally:
            sf.ncell_contract = sf.n ** 3
    return _pair_sums(groups, sf, k_bins, diagonal, block_size)


def _pair_sums(groups, sf, k_bins, diagonal, block_size):
    outs = [DeferredPairSums(specs, k_bins, diagonal) for (_, specs) in groups]
    bs = k_bins if block_size is None else int(block_size)
    blocks = [list(range(b0, min(k_bins, b0 + bs))) for b0 in range(0, k_bins, bs)]
    if diagonal and PAIR_LIST:
        # only the same-bin component pairs are needed: pair-list contraction
        for bi in blocks:
            need = []
            for (_, specs) in groups:
                for ps in specs:
                    need += ps.row_keys(sf, bi) + ps.col_keys(sf, bi)
            sf.release([k for k in list(sf.slot) if k not in set(need)])
            sf.ensure(need)
            for gi, (G, specs) in enumerate(groups):
                pairs = list(dict.fromkeys(kp for ps in specs for b in bi for kp in _entry_keys(ps, sf, b, b)))
                outs[gi].add_pairs(contract_pairs(G, sf, pairs), pairs, bi)
            sf.release_all()
        return outs
    for bi in blocks:
        rows_g = []
        for (_, specs) in groups:
            rk = []
            for ps in specs:
                rk += ps.row_keys(sf, bi)
            rows_g.append(list(dict.fromkeys(rk)))
        col_blocks = [bi] if diagonal else blocks
        for bj in col_blocks:
            cols_g = []
            for (_, specs) in groups:
                ck = []
                for ps in specs:
                    ck += ps.col_keys(sf, bj)
                cols_g.append(list(dict.fromkeys(ck)))
            keep = set().union(*rows_g, *cols_g)
            sf.release([k for k in list(sf.slot) if k not in keep])
            sf.ensure([k for r in rows_g for k in r] + [k for c in cols_g for k in c])
            for idxs in _launch_groups(sf, rows_g, cols_g):
                if len(idxs) == 1:
                    gi = idxs[0]
                    outs[gi].add(contract(groups[gi][0], sf, rows_g[gi], cols_g[gi]), rows_g[gi], cols_g[gi], bi, bj)
                    continue
                Ts = contract_multi([groups[gi][0] for gi in idxs], sf, [rows_g[gi] for gi in idxs],
                                    cols_g[idxs[0]])
                for gi, T in zip(idxs, Ts):
                    outs[gi].add(T, rows_g[gi], cols_g[gi], bi, bj)
        sf.release_all()
    return outs


def _launch_groups(sf, rows_g, cols_g):
    """Groups (weight fields) contracted together: FP32 groups with the same
    columns share one multi-weight launch while rows <= 48, columns <= 24 and
    at most 4 weights; the rest get a launch each."""
    plan = []
    if sf.precision != "f32" or not GRAM_MULTI:
        return [[gi] for gi in range(len(rows_g))]

    def fits(members):
        if GRAM_TC:  # one tensor-core launch: <= 40 rows, <= 24 columns, <= 4 weights
            nr = sum(len(rows_g[j]) for j in members)
            return nr <= 40 and len(cols_g[members[0]]) <= 24 and len(members) <= 4
        # the FFMA launch stages G_0..G_k-1, the padded row window and, unless
        # the columns are a run of the rows inside it, the padded column window;
        # two slab buffers per warp must fit (<= 48 staged rows)
        ridx = [sf.slot[k] for j in members for k in rows_g[j]]
        cidx = [sf.slot[k] for k in cols_g[members[0]]]
        wr, wc = -(-len(ridx) // 8) * 8, -(-len(cidx) // 4) * 4
        shared = any(ridx[o:o + len(cidx)] == cidx and o + wc <= wr for o in range(len(ridx) - len(cidx) + 1))
        return (len(ridx) <= 48 and len(cidx) <= 24 and len(members) <= 4
                and len(members) + wr + (0 if shared else wc) <= 48)

    open_by_cols = {}
    for gi, (rows, cols) in enumerate(zip(rows_g, cols_g)):
        key = tuple(cols)
        cur = open_by_cols.get(key)
        if cur is not None and rows and cols and fits(cur + [gi]):
            cur.append(gi)
            continue
        cur = [gi]
        plan.append(cur)
        open_by_cols[key] = cur
    return plan


def contract_multi(Gs, sf, rows_list, cols):
    """[T_g] with T_g[i, j] = sum_x G_g F_rows_g[i] F_cols[j] (FP64) for FP32
    fields, in one launch (cnpc_contract_gram_multi_g)."""
    ctx = _lib.Context.get()
    ridx, ag = [], []
    for g, rows in enumerate(rows_list):
        ridx += [sf.slot[k] for k in rows]
        ag += [g] * len(rows)
    cidx = [sf.slot[k] for k in cols]
    T = torch.empty((len(ridx), len(cidx)), dtype=torch.float64, device=_device())
    if GRAM_TC:
        ctx.gram_tc_multi_g(sf.ncell_contract, Gs, sf.fields, sf.stride, ridx, ag, cidx, T)
    else:
        ctx.gram_multi_g(sf.ncell_contract, Gs, sf.fields, sf.stride, ridx, ag, cidx, T)
    out, r0 = [], 0
    for rows in rows_list:
        out.append(T[r0:r0 + len(rows)])
        r0 += len(rows)
    return out


# ------------------------------------------------ x = 0 cell of FFT S3 sums
# The FFT S3 source has a spike at x = 0 (the shot-noise constant S W(k) is
# nearly flat in k), where the shell fields also peak.  In FP32 that one
# product dominates the rounding of sum_x src F1 F2, so the FP32 contraction
# runs with the source's x = 0 cell zeroed and the cell's product is added in
# FP64: src(0) = sum_k src(k) and F(0) = sum_{k in bin} conj?(Y(khat)) are mode
# sums evaluated in FP64 from the spectra.

# ------------------------------------------- cross-mock amortisation (opt-in)
# The FFT S3 shells c2r(conj Y_lm * mask_bin) of a unit spectrum, their
# x = 0 values and the bins' mode counts depend only on (nmesh, boxsize, bins,
# lm): with UNIT_SHELL_CACHE they are computed once per shape class and reused
# by later data vectors (one shell class kept at a time).  Off by default:
# every call then computes them, as the reference does.
UNIT_SHELL_CACHE = False
_unit_shells = {}
_unit_origin = {}
_kbin_cache = {}


def clear_unit_shell_cache():
    _unit_shells.clear()
    _unit_origin.clear()
    _kbin_cache.clear()


def unit_shells(n, boxsize, edges, precision, capacity):
    """The persistent unit-spectrum ShellFields of this geometry (UNIT_SHELL_CACHE)."""
    key = (int(n), float(boxsize), tuple(float(e) for e in edges), precision, torch.cuda.current_device())
    sf = _unit_shells.get(key)
    if sf is None or sf.capacity < capacity:
        if _unit_shells:
            torch.cuda.synchronize()  # the old fields may still be read on another stream
        clear_unit_shell_cache()
        sf = ShellFields(n, boxsize, edges, precision, None, None, capacity=capacity)
        sf.persistent = True
        _unit_shells[key] = sf
    return sf


def unit_shell_origin(n, boxsize, edges, precision, legs):
    """{leg: HostCopy of complex F(0) per bin} for unit-spectrum shell legs
    (l, m, 2, conj): F(0) = sum over the bin's full-space modes of Y or conj Y."""
    if UNIT_SHELL_CACHE:
        key = (int(n), float(boxsize), tuple(float(e) for e in edges), precision, tuple(dict.fromkeys(legs)),
               torch.cuda.current_device())
        hit = _unit_origin.get(key)
        if hit is None:
            hit = _unit_origin[key] = _unit_shell_origin(n, boxsize, edges, precision, legs)
        return hit
    return _unit_shell_origin(n, boxsize, edges, precision, legs)


def _unit_shell_origin(n, boxsize, edges, precision, legs):
    ctx = _lib.Context.get()
    code = PRECISION[precision][0]
    unit = ctx.operand(None)
    out = {}
    for leg in dict.fromkeys(legs):
        l, m, src, conj = leg
        if src != 2:
            raise ValueError("origin values are defined for unit-spectrum legs only")
        d = torch.empty(2 * (len(edges) - 1), dtype=torch.float64, device=_device())
        ctx.survey_bins(code, n, float(boxsize), 1, unit, unit, 0.0, angular.harmonic(l, m, True), conj, 1.0,
                        edges, d)
        out[leg] = HostCopy(d)
    return out


def origin_correction(ps, origin, src0, k_bins, diagonal):
    """src(0) F1_i(0) F2_j(0) for one pair spec (k_bins x k_bins, or the diagonal)."""
    def vals(leg):
        v = origin[leg].get()
        return v[0::2] + 1j * v[1::2]

    f1 = vals(ps.leg1)
    if ps.mode == "eq":
        f2 = f1
    elif ps.mode == "conj":
        f2 = ps.sign * np.conj(f1)
    else:
        f2 = vals(ps.leg2)
    if diagonal:
        return src0 * f1 * f2
    return src0 * np.outer(f1, f2)


_DEVICE_BASE = {}


def free_device_bytes():
    """Device memory available to new tensors, without a driver query on the
    hot path (cudaMemGetInfo can stall behind queued work): the driver's free
    memory plus torch's reserved pool, measured once per device, minus what
    torch has allocated since."""
    dev = torch.cuda.current_device()
    base = _DEVICE_BASE.get(dev)
    if base is None:
        free, _ = torch.cuda.mem_get_info()
        base = int(free + torch.cuda.memory_reserved()) - int(torch.cuda.memory_allocated())
        base = (base, int(torch.cuda.memory_allocated()))
        _DEVICE_BASE[dev] = base
    avail, alloc0 = base
    return avail - (int(torch.cuda.memory_allocated()) - alloc0)


def fields_capacity(n, precision, want, reserve_bytes=0, free_bytes=None):
    """How many real n^3 fields fit in the available HBM (leaving headroom).
    ``free_bytes`` (from :func:`free_device_bytes`) spares the driver query."""
    esz = 4 if precision == "f32" else 8
    free = free_device_bytes() if free_bytes is None else int(free_bytes)
    avail = int(free * 0.8) - reserve_bytes
    return max(1, min(int(want), avail // (esz * n ** 3)))
