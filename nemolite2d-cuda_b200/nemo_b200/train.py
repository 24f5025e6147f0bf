"""Training data from the ensemble solver, normalisation, the AdamW training
loop and evaluation of the surrogate against the FP64 solver.

Snapshots are FP32 device tensors [members][H][W][4] (ssh, u west face,
v south face, depth) taken every `every` steps from seeded ensembles of
equal-size members (the batched configuration's recipe at a fixed side).
torch only provides device memory and index gathers; every network kernel
runs in the library.
"""
import math

import numpy as np

from . import SSHN, Ensemble, default_params, generate_members
from .surrogate import adamw, ens_compare

COMMON = dict(dx=1000.0, dy=1000.0, rdt=20.0, cbfr=0.00015, visc=0.1)


def _torch():
    import torch
    return torch


def square_members(seed, n, side, amp_scale):
    ms = generate_members(seed, n, side_min=side, side_max=side, amp_scale=amp_scale)
    for m in ms:
        m.jpi = side
        m.jpj = side
    return ms


def tide_of(member, istp, rdt=20.0):
    """Boundary-row SSH after step istp (original/nemolite2d.f90:629-635)."""
    omega = 2.0 * 3.14159 / (12.42 * 3600.0)
    return member.amp_tide * math.sin(omega * (istp * rdt) + member.tide_phase)


def snapshot_steps(steps, every=10, pair_stride=None):
    """Steps at which generate_runs records snapshots: every `every` steps,
    or with pair_stride the pairs (t, t + every) for t = 0, pair_stride, ...
    (long runs with a bounded number of snapshots)."""
    if not pair_stride:
        return list(range(0, steps + 1, every))
    out = []
    for t in range(0, steps - every + 1, pair_stride):
        out += [t, t + every]
    return out


def generate_runs(sur, seed, nmem, side, steps, every=10, amp_scale=0.2, strict=False,
                  bound=2.5, pair_stride=None, members=None):
    """Runs nmem members from rest for `steps` steps and returns (snaps, tides)
    of the members whose run stays bounded (finite, max |ssh| <= bound x the
    member's tidal amplitude; the reference scheme lets a tide that starts
    rising grow at the corner of the east wall and the open boundary):
    snaps [S][kept][side][side][4] float32 on the device at the steps of
    snapshot_steps(steps, every, pair_stride), tides [S][kept] float32 (the
    boundary SSH at each snapshot's step).  The number of members dropped is
    in generate_runs.dropped.  `members` (a list of side x side members)
    replaces the seeded draw of nmem members."""
    torch = _torch()
    if members is None:
        members = square_members(seed, nmem, side, amp_scale)
    nmem = len(members)
    ens = Ensemble(members, strict=strict, **COMMON)
    at = snapshot_steps(steps, every, pair_stride)
    ns = len(at)
    snaps = torch.empty((ns, nmem, side, side, 4), dtype=torch.float32, device="cuda")
    tides = torch.empty((ns, nmem), dtype=torch.float32)
    istp = 0
    for k in range(ns):
        if at[k] > istp:
            ens.step_n(istp + 1, at[k] - istp)
            istp = at[k]
        torch.cuda.synchronize()
        sur.pack_ens(ens, snaps[k].data_ptr())
        tides[k] = torch.tensor([tide_of(m, istp) for m in members], dtype=torch.float32)
    ens.close()
    amp = torch.tensor([m.amp_tide for m in members], dtype=torch.float32, device="cuda")
    ssh = snaps[..., 0]
    finite = torch.isfinite(snaps).flatten(2).all(2).all(0)
    peak = torch.nan_to_num(ssh.abs(), nan=float("inf")).flatten(2).amax(2).amax(0)
    keep = (finite & (peak <= bound * amp)).nonzero().flatten()
    generate_runs.dropped = nmem - int(keep.numel())
    snaps = snaps.index_select(1, keep)
    tides = tides.cuda().index_select(1, keep)
    torch.cuda.synchronize()
    return snaps, tides


generate_runs.dropped = 0


def generate_dataset(sur, seed, nruns, side, steps, every=10, chunk=256, amp_scale=0.2, bound=2.5):
    """A training set of `nruns` seeded runs of the batched recipe at a fixed
    side (the surrogate-training configuration: 2048 runs of 256 x 256, 500
    steps, snapshots every 10 steps, about 100 GiB of FP32 snapshots),
    generated `chunk` runs at a time, one ensemble per chunk, and kept as one
    snapshot tensor per chunk, so that generation never holds more than one
    chunk twice.  Returns (chunks, dropped): chunks is a list of the
    (snaps, tides) pairs generate_runs returns, dropped the number of runs
    that left the bound."""
    members = square_members(seed, nruns, side, amp_scale)
    chunks, dropped = [], 0
    for c0 in range(0, nruns, chunk):
        snaps, tides = generate_runs(sur, seed, 0, side, steps, every, amp_scale, bound=bound,
                                     members=members[c0:c0 + chunk])
        dropped += generate_runs.dropped
        if snaps.shape[1]:
            chunks.append((snaps, tides))
    return chunks, dropped


def bounded_members(members, steps, common, bound=2.5, checks=2, batch=64, want=None):
    """Indices of the members whose FP64 run from rest stays bounded: finite
    and max |ssh| <= bound x the member's tidal amplitude at `checks` evenly
    spaced points of the run (the last at `steps`).  Screens `batch` members
    per ensemble and stops once `want` members passed (None: screen all)."""
    out = []
    for b0 in range(0, len(members), batch):
        if want is not None and len(out) >= want:
            break
        idx = list(range(b0, min(b0 + batch, len(members))))
        ens = Ensemble([members[i] for i in idx], **common)
        alive = list(range(len(idx)))
        done = 0
        for k in range(1, checks + 1):
            to = steps * k // checks
            ens.step_n(done + 1, to - done)
            done = to
            keep = []
            for i in alive:
                ssh = ens.field(i, SSHN)
                if np.isfinite(ssh).all() and np.abs(ssh).max() <= bound * members[idx[i]].amp_tide:
                    keep.append(i)
            alive = keep
        ens.close()
        out += [idx[i] for i in alive]
    return out


def compute_norm(snaps, paired=False):
    """Input scale/shift per channel and output scale per delta channel from
    a snapshot tensor [S][N][H][W][4] (paired: deltas of the pairs (2i, 2i+1))."""
    torch = _torch()
    sub = snaps[:, ::max(1, snaps.shape[1] // 8)]  # statistics from up to 8 runs
    x = sub.reshape(-1, 4).double()
    mean = x.mean(0)
    std = x.std(0)
    if paired:
        d = (sub[1::2] - sub[0::2]).reshape(-1, 4).double()
    else:
        d = (sub[1:] - sub[:-1]).reshape(-1, 4).double()
    dstd = d.std(0)
    in_shift = [0.0, 0.0, 0.0, float(mean[3])]
    in_scale = [1.0 / max(float(std[c]), 1e-12) for c in range(4)]
    out_scale = [1.0 / max(float(dstd[c]), 1e-12) for c in range(3)]
    del torch
    return in_scale, in_shift, out_scale


class PairSampler:
    """Random (snapshot k, snapshot k+1) pairs of a run set, gathered into
    contiguous device batches; with paired=True only the pairs (2i, 2i+1)
    (runs recorded with a pair_stride)."""

    def __init__(self, snaps, tides, seed=0, paired=False):
        torch = _torch()
        self.snaps, self.tides = snaps, tides
        S, N = snaps.shape[0], snaps.shape[1]
        ks = range(0, S - 1, 2) if paired else range(S - 1)
        self.pairs = [(k, m) for k in ks for m in range(N)]
        self.rng = np.random.default_rng(seed)
        self.order = []
        self.s0 = self.s1 = self.t1 = None
        self._torch = torch

    def batch(self, n):
        torch = self._torch
        if len(self.order) < n:
            self.order = list(self.rng.permutation(len(self.pairs)))
        idx = [self.pairs[self.order.pop()] for _ in range(n)]
        k = torch.tensor([i[0] for i in idx], device="cuda")
        m = torch.tensor([i[1] for i in idx], device="cuda")
        s0 = self.snaps[k, m].contiguous()
        s1 = self.snaps[k + 1, m].contiguous()
        t1 = self.tides[k + 1, m].contiguous()
        torch.cuda.synchronize()
        self.s0, self.s1, self.t1 = s0, s1, t1  # keep alive while the library reads
        return s0, s1, t1


class ChunkPairSampler:
    """Random (snapshot k, snapshot k+1) pairs drawn from a data set held as
    several snapshot tensors (generate_dataset's chunks), gathered into one
    contiguous device batch."""

    def __init__(self, chunks, seed=0):
        torch = _torch()
        self.chunks = chunks
        self.pairs = [(c, k, m) for c, (sn, _) in enumerate(chunks)
                      for k in range(sn.shape[0] - 1) for m in range(sn.shape[1])]
        self.rng = np.random.default_rng(seed)
        self.order = []
        self.s0 = self.s1 = self.t1 = None
        self._torch = torch

    def __len__(self):
        return len(self.pairs)

    def batch(self, n):
        torch = self._torch
        if len(self.order) < n:
            self.order = list(self.rng.permutation(len(self.pairs)))
        idx = [self.pairs[self.order.pop()] for _ in range(n)]
        parts0, parts1, partt = [], [], []
        for c, (sn, td) in enumerate(self.chunks):
            sel = [(k, m) for cc, k, m in idx if cc == c]
            if not sel:
                continue
            k = torch.tensor([i[0] for i in sel], device="cuda")
            m = torch.tensor([i[1] for i in sel], device="cuda")
            parts0.append(sn[k, m])
            parts1.append(sn[k + 1, m])
            partt.append(td[k + 1, m])
        s0 = torch.cat(parts0).contiguous()
        s1 = torch.cat(parts1).contiguous()
        t1 = torch.cat(partt).contiguous()
        torch.cuda.synchronize()
        self.s0, self.s1, self.t1 = s0, s1, t1  # keep alive while the library reads
        return s0, s1, t1


class NoisySampler:
    """Pairs of `base` with Gaussian noise of `sigma` x each field's spread
    added to the input state (ssh, u, v) and the target left the true state
    10 steps on: the network learns to advance a slightly wrong state to the
    right one, which is what it meets after its own earlier calls."""

    def __init__(self, base, sigma, std, seed=0):
        torch = _torch()
        self.base, self.sigma = base, float(sigma)
        self.scale = torch.tensor([float(std[0]), float(std[1]), float(std[2]), 0.0],
                                  dtype=torch.float32, device="cuda") * self.sigma
        self.gen = torch.Generator(device="cuda")
        self.gen.manual_seed(seed)
        self._torch = torch

    def batch(self, n):
        s0, s1, t1 = self.base.batch(n)
        if self.sigma > 0:
            noise = self._torch.randn(s0.shape, generator=self.gen, device="cuda", dtype=self._torch.float32)
            s0 = (s0 + noise * self.scale).contiguous()
            self._torch.cuda.synchronize()
            self.s0 = s0  # keep alive while the library reads
        return s0, s1, t1


def field_std(snaps):
    """Spread of ssh, u, v over a snapshot tensor [S][N][H][W][4] (up to 8 runs)."""
    sub = snaps[:, ::max(1, snaps.shape[1] // 8)]
    x = sub.reshape(-1, 4).double()
    return [float(v) for v in x.std(0)[:3]]


class MixSampler:
    """Batches drawn from several samplers in proportion to `weights`."""

    def __init__(self, samplers, weights, seed=0):
        self.samplers = list(samplers)
        w = np.asarray(weights, dtype=np.float64)
        self.p = w / w.sum()
        self.rng = np.random.default_rng(seed)

    def batch(self, n):
        return self.samplers[int(self.rng.choice(len(self.samplers), p=self.p))].batch(n)


def rollout_runs(sur, seed, nmem, side, windows, k=10, anchor=100, amp_scale=0.2, bound=2.5):
    """Training pairs along hybrid trajectories: members run from rest through
    one solver window, then each window advances by (anchor - k) / k calls of
    the surrogate `sur` followed by k FP64 solver steps, and the pair is (the
    state the surrogate left, the solver's state k steps later) -- the states
    the hybrid controller meets, which carry the surrogate's own errors.
    Returns (snaps, tides) in the paired layout [2*windows][kept][side][side][4]
    of the members that stay bounded; the number dropped is in
    rollout_runs.dropped."""
    torch = _torch()
    members = square_members(seed, nmem, side, amp_scale)
    ens = Ensemble(members, **COMMON)
    snaps = torch.empty((2 * windows, nmem, side, side, 4), dtype=torch.float32, device="cuda")
    tides = torch.empty((2 * windows, nmem), dtype=torch.float32)
    ens.step_n(1, anchor)
    istp = anchor
    for w in range(windows):
        for _ in range((anchor - k) // k):
            sur.advance_ens(ens, istp + k)
            istp += k
        torch.cuda.synchronize()
        sur.pack_ens(ens, snaps[2 * w].data_ptr())
        tides[2 * w] = torch.tensor([tide_of(m, istp) for m in members], dtype=torch.float32)
        ens.step_n(istp + 1, k)
        istp += k
        torch.cuda.synchronize()
        sur.pack_ens(ens, snaps[2 * w + 1].data_ptr())
        tides[2 * w + 1] = torch.tensor([tide_of(m, istp) for m in members], dtype=torch.float32)
    ens.close()
    amp = torch.tensor([m.amp_tide for m in members], dtype=torch.float32, device="cuda")
    finite = torch.isfinite(snaps).flatten(2).all(2).all(0)
    peak = torch.nan_to_num(snaps[..., 0].abs(), nan=float("inf")).flatten(2).amax(2).amax(0)
    keep = (finite & (peak <= bound * amp)).nonzero().flatten()
    rollout_runs.dropped = nmem - int(keep.numel())
    snaps = snaps.index_select(1, keep)
    tides = tides.cuda().index_select(1, keep)
    torch.cuda.synchronize()
    return snaps, tides


rollout_runs.dropped = 0


def train(sur, sampler, iters, batch, lr=1e-3, weight_decay=1e-4, lr_min=1e-5, log_every=0):
    """AdamW with cosine learning-rate decay; returns the loss history."""
    losses = []
    for it in range(iters):
        c = 0.5 * (1.0 + math.cos(math.pi * it / max(iters, 1)))
        hp = adamw(lr=lr_min + (lr - lr_min) * c, weight_decay=weight_decay)
        s0, s1, t1 = sampler.batch(batch)
        losses.append(sur.train_step(s0.data_ptr(), s1.data_ptr(), t1.data_ptr(), batch, hp))
        if log_every and (it % log_every == 0 or it == iters - 1):
            print("iter %5d  loss %.5f  lr %.2e" % (it, losses[-1], hp.lr), flush=True)
    return losses


def rel_l2(a, b):
    """sqrt(sum (a-b)^2 / sum b^2) per leading index (torch tensors)."""
    d = ((a - b).double() ** 2).flatten(1).sum(1)
    r = (b.double() ** 2).flatten(1).sum(1)
    return (d / r.clamp_min(1e-300)).sqrt()


def evaluate_one_call(sur, seed, nmem, side, spin_up, amp_scale=0.2):
    """Relative SSH/u/v L2 errors after one 10-step surrogate call from the
    FP64 state after spin_up steps, against the FP64 solver, for the
    surrogate and for persistence (no change).  nmem <= the surrogate's
    batch.  Returns dict of (nmem, 3) arrays."""
    torch = _torch()
    members = square_members(seed, nmem, side, amp_scale)
    a = Ensemble(members, **COMMON)
    b = Ensemble(members, **COMMON)
    a.step_n(1, spin_up)
    b.step_n(1, spin_up)
    s0 = torch.empty((nmem, side, side, 4), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    sur.pack_ens(a, s0.data_ptr())
    sur.advance_ens(a, spin_up + 10)    # surrogate call
    b.step_n(spin_up + 1, 10)           # FP64 solver
    sur_err = ens_compare(a, b)
    s1 = torch.empty_like(s0)
    sur.pack_ens(b, s1.data_ptr())
    torch.cuda.synchronize()
    pers = torch.stack([rel_l2(s0[..., c], s1[..., c]) for c in range(3)], 1).cpu().numpy()
    a.close()
    b.close()
    return {"surrogate": sur_err, "persistence": pers}
