"""Distributed C2C transforms over several GPUs (one process per GPU).

FFTND is the reference's multi-rank FFTND: commDims = [P_0, ..., P_{nda-1},
1, ..., 1] distributes the leading nda axes over a Cartesian process grid
(one axis: slabs; several: pencils), src/cpp/slab_nd.cpp:71-254 and
shafft_internal.cpp:62-127, 229-381.  torch.distributed carries the
exchanges (NCCL between GPUs; a gloo group exchanges through host memory);
everything on the device goes through the kernel library:

  stage 0        the leading nda axes block-partitioned over the grid
  subplan s      transforms the contiguous axes not yet transformed
                 (shafft_sm100_plan_create_axes on the local block)
  exchange i     inside the grid line of cart dimension nda-1-i: the
                 distributed axis b of that slot becomes contiguous and the
                 contiguous axis a = b + nca (nca = ndim - nda) becomes
                 distributed -- pack the local block along a into per-peer
                 blocks, all-to-all, unpack along b (skipped when b is the
                 outermost axis).  The pack is fused into the stores of the
                 subplan before the exchange and the unpack into the loads of
                 the subplan after it where the kernel library can
                 (shafft_sm100_plan_create_axes_mapped: power-of-two shapes
                 whose neighbouring step is an out-of-place specialised pass);
                 otherwise they are separate kernels
                 (shafft_sm100_pack_blocks / shafft_sm100_unpack_blocks)
  sequences      subplans alternate with ceil(nda / nca) sequences of up to
                 nca exchanges; after the last one the layout is
                 REDISTRIBUTED (TransformLayout INITIAL replays the exchanges
                 backwards); backward runs the same steps in reverse

with the reference's block partition (the first n % P parts one element
longer, detail/partition.hpp:40-44), buffer-swap contract (the result is in
the buffer get_buffers() reports as data) and (1/sqrt(N))^k normalisation.
Methods return the reference's status codes.  Ranks beyond prod(commDims)
are inactive: they own no data and belong to no grid line.  FFT1D (below) is
the reference's distributed 1-D transform (the P x P four-step path, and
Bluestein over it for lengths P^2 does not divide).
"""
from __future__ import annotations

import ctypes
import itertools
import math

from . import (BACKWARD, C2C, ERR_ALLOC, ERR_DIM_MISMATCH, ERR_INVALID_DECOMP, ERR_INVALID_DIM,
               ERR_INVALID_FFTTYPE, ERR_INVALID_LAYOUT, ERR_INVALID_STATE, ERR_NO_BUFFER,
               ERR_NOT_IMPL, ERR_NULLPTR, ERR_PLAN_NOT_INIT, FORWARD, LAYOUT_INITIAL,
               LAYOUT_REDISTRIBUTED, TENSOR_LAYOUT_CURRENT, TENSOR_LAYOUT_INITIAL,
               TENSOR_LAYOUT_REDISTRIBUTED, Z2Z)


def block_partition(total: int, nparts: int, rank: int):
    """(local length, local start) of `rank`'s block; the first total % nparts
    blocks are one element longer."""
    q, r = divmod(total, nparts)
    return (q + 1, rank * (q + 1)) if rank < r else (q, r * (q + 1) + (rank - r) * q)


# ---- decomposition search (the reference's configurationND) ---------------
# src/cpp/configuration.cpp:94-600, restated: a user grid is validated
# (configurationCart); a requested number of distributed axes is tried
# exactly; otherwise d = ndim-1 .. 1 (MAXIMIZE_NDA) or 1 .. ndim-1
# (MINIMIZE_NDA) is tried: a balanced grid of the world size (as
# MPI_Dims_create), capped per axis by min(size[i], size[i + ndim - d]),
# packed greedily into the leading axes (factors fill an axis up to its cap
# before spilling to the next), accepted when every active rank's block
# passes the 32-bit element limit and the memory limit (two buffers).  Every
# rank's block is computed locally, so no reduction across ranks is needed.

MAXIMIZE_NDA, MINIMIZE_NDA = 0, 1


def _dims_create(n, d):
    """Balanced factorisation of n into d factors, non-increasing (the
    result MPI_Dims_create gives for an all-zero dims array)."""
    primes, m, f = [], n, 2
    while f * f <= m:
        while m % f == 0:
            primes.append(f)
            m //= f
        f += 1
    if m > 1:
        primes.append(m)
    dims = [1] * d
    for p in sorted(primes, reverse=True):
        i = dims.index(min(dims))
        dims[i] *= p
    return sorted(dims, reverse=True)


def _min_caps(ndim, d, sizes):
    return [min(sizes[i], sizes[i + ndim - d]) for i in range(d)]


def _largest_divisor_leq(n, limit):
    if n <= 1 or limit < 2:
        return 1
    return max(x for x in range(1, min(n, limit) + 1) if n % x == 0)


def _pack_prefix_with_spill(ndim, grid, sizes, caps):
    factors = [g for g in grid if g > 1]
    grid[:] = [1] * ndim
    max_axes = max(0, ndim - 1)
    cap_left = [max(1, min(sizes[i], caps[i]) if caps and i < len(caps) else sizes[i])
                for i in range(max_axes)]
    axis = 0
    for f in factors:
        rem = f
        while rem > 1 and axis < max_axes:
            room = cap_left[axis] // grid[axis]
            if room < 2:
                axis += 1
                continue
            used = _largest_divisor_leq(rem, room)
            if used <= 1:
                axis += 1
                continue
            grid[axis] *= used
            rem //= used
            if grid[axis] == cap_left[axis]:
                axis += 1
    dp = 0
    while dp < max_axes and grid[dp] > 1:
        dp += 1
    for i in range(dp, ndim):
        grid[i] = 1
    return dp


def _blocks_ok(dims, d, grid, precision, mem_limit):
    """Every active rank's block within the 32-bit element limit and the
    memory limit (two buffers of the local block)."""
    ndim = len(dims)
    esize = 8 if precision == C2C else 16
    for rank in range(math.prod(grid[:d]) if d else 1):
        coords, r = [], rank
        for g in reversed(grid[:d]):
            coords.insert(0, r % g)
            r //= g
        sub = list(dims)
        for i in range(d):
            sub[i] = block_partition(dims[i], grid[i], coords[i])[0]
        n = math.prod(sub)
        if min(sub) <= 0 or n > 2 ** 31 - 1:
            return False
        if mem_limit and 2 * esize * n > mem_limit:
            return False
    return True


def configuration_nd(dims, world, rank=0, precision=C2C, comm_dims=None, nda=0,
                     strategy=MAXIMIZE_NDA, mem_limit=0):
    """(status, commDims, nda, subsize, offset, active ranks) for `world`
    ranks, as the reference's shafft::configurationND
    (src/cpp/configuration.cpp:530-600)."""
    ndim = len(dims)
    sizes = [int(x) for x in dims]
    grid = [int(c) for c in (comm_dims or [0] * ndim)]
    if len(grid) != ndim:
        return ERR_DIM_MISMATCH, None, 0, None, None, 0

    def result(g, d):
        L = SlabLayout(sizes, g, rank)
        act = math.prod(g[:d]) if d else 1
        return 0, list(g), d, list(L.sub[0]), list(L.off[0]), act

    if any(grid) and all(c > 0 for c in grid):  # a user grid (configurationCart)
        d = 0
        while d < ndim and grid[d] > 1:
            d += 1
        ok = d < ndim and all(c == 1 for c in grid[d:])
        if d == 0:
            ok = world == 1
        if ok and d:
            caps = _min_caps(ndim, d, sizes)
            ok = all(1 <= grid[i] <= min(sizes[i], caps[i]) for i in range(d)) and math.prod(grid[:d]) <= world
        if ok and _blocks_ok(sizes, d, grid, precision, mem_limit):
            return result(grid, d)

    def try_d(d, strict):
        if d < 1 or d > ndim - 1:
            return None
        g = [1] * ndim
        caps = _min_caps(ndim, d, sizes)
        if d == 1:
            g[0] = min(world, sizes[0])
        else:
            md = _dims_create(world, d)
            for i in range(d):
                g[i] = max(1, min(md[i], caps[i]))
        if strict and sum(1 for i in range(d) if g[i] > 1) != d:
            return None
        de = d
        if not strict:
            de = _pack_prefix_with_spill(ndim, g, sizes, caps)
            if de == 0 and world > 1:
                return None
            if de != d:
                caps2 = _min_caps(ndim, de, sizes)
                if any(g[i] > caps2[i] for i in range(de)):
                    return None
        if not _blocks_ok(sizes, de, g, precision, mem_limit):
            return None
        return g, de

    if nda > 0:
        r = try_d(nda, True)
        return result(*r) if r else (ERR_INVALID_DECOMP, None, 0, None, None, 0)
    order = range(ndim - 1, 0, -1) if strategy == MAXIMIZE_NDA else range(1, ndim)
    for d in order:
        r = try_d(d, False)
        if r:
            return result(*r)
    if world == 1:
        return result([1] * ndim, 0)
    return ERR_INVALID_DECOMP, None, 0, None, None, 0


class SlabLayout:
    """Index bookkeeping of the decomposition (pure host arithmetic): the
    distributed / contiguous axes, local block (subsize, offset) of every
    exchange index 0..nda, the exchanges' axes and grid dimensions, and the
    exchange sequences with the axes each subplan transforms."""

    def __init__(self, dims, comm_dims, rank: int):
        self.dims = tuple(int(d) for d in dims)
        self.comm_dims = [int(c) for c in comm_dims]
        d = len(self.dims)
        nda = 0
        for c in self.comm_dims:
            if c > 1:
                nda += 1
            else:
                break
        self.nda, self.nca = nda, d - nda
        self.grid = self.comm_dims[:nda]
        self.P = math.prod(self.grid) if nda else 1
        self.rank = int(rank)
        self.active = self.rank < self.P
        # cart coordinates, row-major over the grid (MPI_Cart_create, no reorder)
        self.coords, r = [], self.rank
        for g in reversed(self.grid):
            self.coords.insert(0, r % g if self.active else 0)
            r //= g
        das, cas = [list(range(nda))], [list(range(nda, d))]
        self.axes_a, self.axes_b = [], []
        for i in range(nda):
            da, ca = list(das[-1]), list(cas[-1])
            b = da[nda - i - 1]
            a = b + self.nca
            da[nda - i - 1] = a
            ca[ca.index(a)] = b
            das.append(da)
            cas.append(ca)
            self.axes_a.append(a)
            self.axes_b.append(b)
        self.das, self.cas = das, cas
        self.sub, self.off = [], []
        for s in range(nda + 1):
            sub, off = list(self.dims), [0] * d
            for j in range(nda):
                ax = das[s][j]
                n, st = block_partition(self.dims[ax], self.grid[j], self.coords[j]) if self.active else (0, 0)
                sub[ax], off[ax] = n, st
            self.sub.append(sub)
            self.off.append(off)
        nes = -(-nda // self.nca) if nda else 0
        self.es = [min(self.nca, nda - i * self.nca) for i in range(nes)]
        done, self.tf_axes, self.plan_index = set(), [], []
        for s in range(nes + 1):
            idx = sum(self.es[:s])
            ta = [a for a in cas[idx] if a not in done]
            done.update(ta)
            self.tf_axes.append(ta)
            self.plan_index.append(idx)

    def size(self, idx: int) -> int:
        return math.prod(self.sub[idx]) if self.active else 0

    def alloc_size(self) -> int:
        return max(self.size(s) for s in range(self.nda + 1))

    def grid_line(self, j):
        """World ranks of this rank's grid line along cart dimension j."""
        out = []
        for c in range(self.grid[j]):
            co = list(self.coords)
            co[j] = c
            r = 0
            for g, x in zip(self.grid, co):
                r = r * g + x
            out.append(r)
        return out

    def exchange(self, i):
        """Exchange i (stage i -> i+1): (cart dim, axis a, axis b, Q,
        pack geometry of stage i along a, unpack geometry of stage i+1 along
        b, send counts, receive counts); the backward exchange swaps roles."""
        j = self.nda - i - 1
        a, b = self.axes_a[i], self.axes_b[i]
        Q = self.grid[j]
        sa, sb = self.sub[i], self.sub[i + 1]
        pack = (math.prod(sa[:a]), self.dims[a], math.prod(sa[a + 1:]))
        unpack = (math.prod(sb[:b]), self.dims[b], math.prod(sb[b + 1:]))
        per_a = self.size(i) // self.dims[a] if self.active else 0
        per_b = self.size(i + 1) // self.dims[b] if self.active else 0
        send = [per_a * block_partition(self.dims[a], Q, q)[0] for q in range(Q)]
        recv = [per_b * block_partition(self.dims[b], Q, q)[0] for q in range(Q)]
        return j, a, b, Q, pack, unpack, send, recv


class FFTND:
    """Distributed shafft::FFTND over a torch.distributed process group;
    buffers are torch CUDA tensors of at least alloc_size() complex
    elements."""

    def __init__(self):
        self._state = "created"
        self.norm_exponent = 0

    # lifecycle -------------------------------------------------------------
    def init(self, comm_dims, dims, precision=C2C, group=None,
             output_policy=LAYOUT_REDISTRIBUTED, device_ops=None) -> int:
        """Validation follows planNDConfigure (src/cpp/shafft_internal.cpp:229-333)."""
        import torch.distributed as dist
        if self._state != "created":
            return ERR_INVALID_STATE
        dims = [int(x) for x in dims]
        comm_dims = [int(x) for x in comm_dims]
        if len(dims) < 1:
            return ERR_INVALID_DIM
        if len(comm_dims) != len(dims):
            return ERR_DIM_MISMATCH
        if precision not in (C2C, Z2Z):
            return ERR_INVALID_FFTTYPE
        if output_policy not in (LAYOUT_REDISTRIBUTED, LAYOUT_INITIAL):
            return ERR_INVALID_LAYOUT
        ndim = len(dims)
        if comm_dims[-1] != 1 or any(c < 1 or c > n for c, n in zip(comm_dims, dims)):
            return ERR_INVALID_DECOMP
        nda = 0
        for c in comm_dims:
            if c > 1:
                nda += 1
            else:
                break
        if any(c > 1 for c in comm_dims[nda:]):
            return ERR_INVALID_DECOMP
        nca = ndim - nda
        # cross-axis rule: grid dimension j later partitions axis j + nca
        if any(comm_dims[j] > dims[j + nca] for j in range(nda)):
            return ERR_INVALID_DECOMP
        world = dist.get_world_size(group) if dist.is_initialized() else 1
        rank = dist.get_rank(group) if dist.is_initialized() else 0
        if ndim == 1 and world > 1:
            return ERR_INVALID_DECOMP
        if math.prod(comm_dims[:nda] or [1]) > world:
            return ERR_INVALID_DECOMP
        self.dims, self.precision, self.group = tuple(dims), precision, group
        self.output_policy = output_policy
        self.world, self.rank = world, rank
        self.layout = SlabLayout(dims, comm_dims, rank)
        # one process group per grid line (created by every rank, same order)
        self.lines = {}
        if self.layout.nda and world > 1:
            L = self.layout
            for j in range(L.nda):
                others = [range(g) for k, g in enumerate(L.grid) if k != j]
                for rest in itertools.product(*others):
                    members = []
                    for c in range(L.grid[j]):
                        co = list(rest)
                        co.insert(j, c)
                        r = 0
                        for g, x in zip(L.grid, co):
                            r = r * g + x
                        members.append(r)
                    grp = dist.new_group(members) if len(members) < world else group
                    if L.active and members == L.grid_line(j):
                        self.lines[j] = grp
        self.ops = device_ops
        self.stage = 0
        self._state = "configured"
        return 0

    def plan(self) -> int:
        if self._state == "created":
            return ERR_PLAN_NOT_INIT
        if self._state != "configured":
            return ERR_INVALID_STATE
        if self.ops is None:
            self.ops = CudaOps(self.precision)
        L = self.layout
        self.subplans = []
        self._variants = {}
        if L.active:
            for s, idx in enumerate(L.plan_index):
                self.subplans.append(self.ops.plan(L.sub[idx], L.tf_axes[s]))
            # subplans with the neighbouring exchanges' packing fused, for
            # every execute sequence the output policy leads to
            starts = [(FORWARD, 0), (BACKWARD, L.nda)]
            if self.output_policy == LAYOUT_INITIAL:
                starts.append((BACKWARD, 0))
            for direction, stage in starts:
                seq = self._sequence(direction, stage)
                for pos, op in enumerate(seq):
                    if op[0] == "fft":
                        self._variant(op[1], *self._maps(seq, pos))
        self.data = self.work = None
        self._state = "planned"
        return 0

    def release(self):
        for p in getattr(self, "subplans", []):
            self.ops.destroy(p)
        for v in getattr(self, "_variants", {}).values():
            if v is not None:  # None: nothing was fused, the plain subplan served
                self.ops.destroy(v[0])
        self.subplans = []
        self._variants = {}
        self._state = "released"

    # buffers ---------------------------------------------------------------
    def alloc_size(self) -> int:
        return self.layout.alloc_size() if self._state in ("configured", "planned") else 0

    def set_buffers(self, data, work) -> int:
        if self._state != "planned":
            return ERR_PLAN_NOT_INIT
        if self.layout.active:
            if data is None or work is None:
                return ERR_NULLPTR
            n = self.alloc_size()
            if data.numel() < n or work.numel() < n or data.data_ptr() == work.data_ptr():
                return ERR_ALLOC
        self.data, self.work = data, work
        return 0

    def get_buffers(self):
        return 0, self.data, self.work

    # layout queries (shafft.hpp:252-265) -------------------------------------
    def _index_of(self, which):
        if which == TENSOR_LAYOUT_CURRENT:
            return self.stage
        if which == TENSOR_LAYOUT_INITIAL:
            return 0
        if which == TENSOR_LAYOUT_REDISTRIBUTED:
            return self.layout.nda
        return None

    def get_layout(self, which=TENSOR_LAYOUT_CURRENT):
        s = self._index_of(which)
        if s is None:
            return ERR_INVALID_LAYOUT, [], []
        return 0, list(self.layout.sub[s]), list(self.layout.off[s])

    def get_axes(self, which=TENSOR_LAYOUT_CURRENT):
        s = self._index_of(which)
        if s is None:
            return ERR_INVALID_LAYOUT, [], []
        return 0, list(self.layout.cas[s]), list(self.layout.das[s])

    # compute ---------------------------------------------------------------
    def _sequence(self, direction, stage):
        """The steps of one execute that starts at `stage`, in order:
        ("fft", s) runs subplan s; ("x", i, forward) is exchange i (stage i
        <-> i + 1) in that direction."""
        L = self.layout
        nes, seq = len(L.es), []
        if direction == FORWARD:
            for s in range(nes + 1):
                seq.append(("fft", s))
                if s < nes:
                    for _ in range(L.es[s]):
                        seq.append(("x", stage, True))
                        stage += 1
            if self.output_policy == LAYOUT_INITIAL:
                while stage > 0:
                    seq.append(("x", stage - 1, False))
                    stage -= 1
        else:
            while stage < L.nda:  # re-apply the redistribution first
                seq.append(("x", stage, True))
                stage += 1
            for s in range(nes, -1, -1):
                seq.append(("fft", s))
                if s > 0:
                    for _ in range(L.es[s - 1]):
                        seq.append(("x", stage - 1, False))
                        stage -= 1
        return seq

    def _geometry(self, i, forward):
        """(cart dim, parts, pack, unpack, send, recv) of exchange i in a
        direction; pack / unpack = (outer, n, inner) of the block layout."""
        j, a, b, Q, pack, unpack, send, recv = self.layout.exchange(i)
        if not forward:
            pack, unpack, send, recv = unpack, pack, recv, send
        return j, Q, pack, unpack, send, recv

    def _maps(self, seq, pos):
        """Block maps to fuse into the subplan at seq[pos]: the unpack of the
        exchange before it (its loads) and the pack of the exchange after it
        (its stores), each (outer, n, inner, parts) or None when that side
        needs no (un)packing."""
        load = store = None
        if pos > 0 and seq[pos - 1][0] == "x":
            _, Q, _, unpack, _, _ = self._geometry(*seq[pos - 1][1:])
            if unpack[0] != 1:
                load = tuple(unpack) + (Q,)
        if pos + 1 < len(seq) and seq[pos + 1][0] == "x":
            _, Q, pack, _, _, _ = self._geometry(*seq[pos + 1][1:])
            if pack[0] != 1:
                store = tuple(pack) + (Q,)
        return load, store

    def _variant(self, s, load, store):
        """(plan handle, fused bits) of subplan s with the maps fused where
        the library can (bit 0: load, bit 1: store); the plain subplan when
        there is nothing to fuse."""
        if (load is None and store is None) or not hasattr(self.ops, "plan_mapped"):
            return self.subplans[s], 0
        key = (s, load, store)
        if key not in self._variants:
            L = self.layout
            idx = L.plan_index[s]
            h, fused = self.ops.plan_mapped(L.sub[idx], L.tf_axes[s], load, store)
            if fused == 0:
                self.ops.destroy(h)
                h = self.subplans[s]
                self._variants[key] = None
                return h, 0
            self._variants[key] = (h, fused)
        v = self._variants[key]
        return (self.subplans[s], 0) if v is None else v

    def _fft(self, s, direction, load=None, store=None):
        h, fused = self._variant(s, load, store)
        self.ops.execute(h, self.data, self.work, direction)
        self.data, self.work = self.work, self.data
        return fused

    def _exchange(self, i, forward, packed=False, leave_blocks=False):
        """Exchange i in a direction; the result is left in data.  packed:
        data already holds the per-peer blocks (the subplan before stored
        them); leave_blocks: the received blocks stay unpacked (the subplan
        after loads them through its map)."""
        j, Q, pack, unpack, send, recv = self._geometry(i, forward)
        grp = self.lines.get(j, self.group)
        if pack[0] == 1 or packed:  # outermost-axis blocks are row ranges already
            src = self.data
        else:
            self.ops.pack(self.data, self.work, *pack, Q)
            src = self.work
        dst = self.work if src is self.data else self.data
        self.ops.alltoall(dst, src, recv, send, grp, Q)
        if unpack[0] == 1 or leave_blocks:
            if dst is not self.data:
                self.data, self.work = self.work, self.data
        else:
            out = self.work if dst is self.data else self.data
            self.ops.unpack(dst, out, *unpack, Q)
            if out is not self.data:
                self.data, self.work = self.work, self.data
        self.stage = i + 1 if forward else i

    def execute(self, direction) -> int:
        if self._state != "planned":
            return ERR_PLAN_NOT_INIT
        L = self.layout
        if not L.active:
            self.norm_exponent += 1
            return 0
        if self.data is None or self.work is None:
            return ERR_NO_BUFFER
        if direction not in (FORWARD, BACKWARD):
            return ERR_INVALID_STATE
        seq = self._sequence(direction, self.stage)
        # which subplans load / store the block layouts of their neighbours
        fused = [0] * len(seq)
        for pos, op in enumerate(seq):
            if op[0] == "fft":
                fused[pos] = self._variant(op[1], *self._maps(seq, pos))[1]
        for pos, op in enumerate(seq):
            if op[0] == "fft":
                self._fft(op[1], direction, *self._maps(seq, pos))
            else:
                packed = pos > 0 and seq[pos - 1][0] == "fft" and bool(fused[pos - 1] & 2)
                leave = pos + 1 < len(seq) and seq[pos + 1][0] == "fft" and bool(fused[pos + 1] & 1)
                self._exchange(op[1], op[2], packed, leave)
        self.norm_exponent += 1
        return 0

    def normalize(self) -> int:
        """data *= (1/sqrt(N))^k, k = executes since the last normalize."""
        if self._state != "planned":
            return ERR_PLAN_NOT_INIT
        if self.norm_exponent and self.layout.active:
            f = (1.0 / math.sqrt(math.prod(self.dims))) ** self.norm_exponent
            self.ops.scale(self.data, self.layout.size(self.stage), f)
        self.norm_exponent = 0
        return 0


def select_path_1d(n: int, nranks: int):
    """(path, fft_length, local_size) of a distributed 1-D transform of n
    points on nranks ranks: the reference's selectPath with its default
    padding rule (src/cpp/fft/hipfft_method/1d/fft1d_path_selector.hpp:30-107,
    fft1d_handle.hpp:16-22, padding not allowed).  The P x P four-step runs
    when P^2 divides n; otherwise Bluestein, whose convolution length M is
    2n - 1 rounded up to a multiple of P^2."""
    p2 = nranks * nranks
    if n % p2 == 0:
        return "cooley_tukey", n, n // nranks
    m = -(-(2 * n - 1) // p2) * p2
    return "bluestein", m, m // nranks


def _block_1d(n: int, size: int, rank: int):
    """(local_n, local_start) of rank in blocks of `size` over n points, the
    start clamped to n (fft1d_method.hip:96-106)."""
    off = rank * size
    return (min(size, n - off) if off < n else 0), min(off, n)


def configuration_1d(n: int, world: int, rank: int):
    """(local_n, local_start, local_alloc, active_ranks): the reference's
    fft1dQueryLayout (fft1d_method.hip:329-414).  The path chosen for all
    `world` ranks gives the block size; ranks whose block is empty are
    inactive (all zeros); the path is then chosen again for the active ranks
    0 .. active_ranks-1, whose blocks (input and output alike) follow."""
    _, _, l0 = select_path_1d(n, world)
    active = min(world, -(-n // l0))
    if rank * l0 >= n:
        return 0, 0, 0, active
    _, _, l = select_path_1d(n, active)
    ln, ls = _block_1d(n, l, rank)
    return ln, ls, l, active


class FFT1D:
    """Distributed shafft::FFT1D over a torch.distributed group.  The layout
    is configuration_1d's: ranks 0 .. A-1 are active and rank r holds
    x[r*L, r*L + local_n) in a buffer of L elements (the same block before
    and after a transform); the other ranks are inactive and every call on
    them returns 0 without work.  The active ranks form their own process
    group (created by every rank of the group, in the same order).

    Path A (A^2 divides N; src/cpp/fft/hipfft_method/1d/
    fft1d_cooley_tukey_executor.hip:175-290), the A x A four-step over
    F = N points with L = F/A and C = L/A:

      1. all-to-all of C-element chunks      -> [s][c] = x[s*L + r*C + c]
      2. length-A DFTs over s (one column pass of an [A][C] plan)
                                              -> [k1][c], already the send order
      3. twiddle w_F^{(r*C + c) k1}           (shafft_sm100_twiddle_rows)
      4. all-to-all                           -> [s][c] = column r*... of k1 = r
      5. length-L DFT                         -> X[r + A*k2] at k2
      6. all-to-all of the C-chunks of k2     -> [s][j] = X[r*L + s + A*j]
      7. [A][C] -> [C][A] transpose           (shafft_sm100_unpack_blocks)

    Path B (otherwise; 1d/fft1d_bluestein_executor.hip:209-448): Bluestein
    with the four-step above over the convolution length F = M.  At plan
    time each rank generates its blocks of the chirp b and of the kernel v
    (shafft_sm100_bluestein_chirps) and transforms v; an execute modulates
    (conjugating the input for a backward transform), runs the forward
    four-step, multiplies by the kernel's spectrum, runs the backward
    four-step, and scales by 1/M while demodulating (conjugating the output
    for a backward transform) -- all through shafft_sm100_chirp_multiply.

    The result is in the buffer get_buffers() reports as data (the buffers
    swap on every execute, Slab1D::swapBuffers)."""

    def __init__(self):
        self._state = "created"
        self.norm_exponent = 0

    def init(self, n, local_n, local_start, precision=C2C, group=None, device_ops=None) -> int:
        import torch.distributed as dist
        if self._state != "created":
            return ERR_INVALID_STATE
        if precision not in (C2C, Z2Z):
            return ERR_INVALID_FFTTYPE
        n, local_n, local_start = int(n), int(local_n), int(local_start)
        if n < 1:
            return ERR_INVALID_DIM
        world = dist.get_world_size(group) if dist.is_initialized() else 1
        r = dist.get_rank(group) if dist.is_initialized() else 0
        ln, ls, la, active = configuration_1d(n, world, r)
        if (local_n, local_start) != (ln, ls):
            return ERR_INVALID_DECOMP
        # the active ranks' group (every rank of `group` takes part)
        sub = group
        if world > 1 and active < world:
            ranks = list(range(active))
            if group is not None:
                ranks = [dist.get_global_rank(group, x) for x in ranks]
            sub = dist.new_group(ranks)
        self.active = r < active
        self.N, self.precision, self.ops = n, precision, device_ops
        self.A, self.rank, self.local_n, self.local_start = active, r, ln, ls
        self.path, self.F, self.L = select_path_1d(n, active)
        self.C = self.L // active
        self.group = sub if self.active else None
        self._state = "configured"
        return 0

    def plan(self) -> int:
        if self._state == "created":
            return ERR_PLAN_NOT_INIT
        if self._state != "configured":
            return ERR_INVALID_STATE
        self.plans = []
        self.data = self.work = self.scratch = None
        if self.active:
            if self.ops is None:
                self.ops = CudaOps(self.precision)
            if self.A == 1:
                self.plans = [self.ops.plan([self.N], [0])]
            else:
                self.plans = [self.ops.plan([self.A, self.C], [0]), self.ops.plan([self.L], [0])]
            if self.path == "bluestein":
                L, ops = self.L, self.ops
                self.chirp = ops.empty(L)
                self.vhat = ops.empty(L)
                self.mbuf = [ops.empty(L), ops.empty(L), ops.empty(L)]
                ops.chirps(self.chirp, None, self.N, self.F, self.local_start, self.rank * L, L)
                ops.chirps(None, self.mbuf[0], self.N, self.F, self.local_start, self.rank * L, L)
                self._four_step(self.mbuf[0], self.vhat, self.mbuf[1], FORWARD)
        self._state = "planned"
        return 0

    def release(self):
        for h in getattr(self, "plans", []):
            self.ops.destroy(h)
        self.plans = []
        self.chirp = self.vhat = None
        self.mbuf = []
        self._state = "released"

    def alloc_size(self) -> int:
        return self.L if self._state in ("configured", "planned") and self.active else 0

    def get_layout(self):
        """(status, local_n, local_start): the same block before and after a
        transform (fft1d_method.hip:396-397)."""
        if self._state not in ("configured", "planned"):
            return ERR_PLAN_NOT_INIT, 0, 0
        return 0, self.local_n, self.local_start

    def set_buffers(self, data, work) -> int:
        if self._state != "planned":
            return ERR_PLAN_NOT_INIT
        if not self.active:  # inactive ranks may pass nothing
            self.data, self.work = data, work
            return 0
        if data is None or work is None:
            return ERR_NULLPTR
        if data.numel() < self.L or work.numel() < self.L or data.data_ptr() == work.data_ptr():
            return ERR_ALLOC
        self.data, self.work = data, work
        self.scratch = data.new_empty(self.L)  # plan-owned, as the reference's dBuf/dTemp
        return 0

    def get_buffers(self):
        return 0, self.data, self.work

    def _four_step(self, x, w, s, direction):
        """Steps 1-7 of the class docstring over F points; x and s are
        clobbered, the result lands in w."""
        ops, A, C = self.ops, self.A, self.C
        if A == 1:
            ops.execute(self.plans[0], x, w, direction)
            return
        eq = [C] * A
        ops.alltoall(w, x, eq, eq, self.group, A)                   # 1
        ops.execute(self.plans[0], w, s, direction)                 # 2  [k1][c]
        ops.twiddle(s, A, C, self.rank * C, self.F, -1 if direction == FORWARD else 1)  # 3
        ops.alltoall(x, s, eq, eq, self.group, A)                   # 4
        ops.execute(self.plans[1], x, s, direction)                 # 5  X[r + A k2]
        ops.alltoall(x, s, eq, eq, self.group, A)                   # 6  [s][j]
        ops.unpack(x, w, C, A, 1, A)                                # 7  [j][s]

    def execute(self, direction) -> int:
        if self._state != "planned":
            return ERR_PLAN_NOT_INIT
        if direction not in (FORWARD, BACKWARD):
            return ERR_INVALID_STATE
        if not self.active:
            self.norm_exponent += 1
            return 0
        if self.data is None:
            return ERR_NO_BUFFER
        x, w = self.data, self.work
        if self.path == "cooley_tukey":
            self._four_step(x, w, self.scratch, direction)
        else:
            ops, L, (m0, m1, m2) = self.ops, self.L, self.mbuf
            back = 1 if direction == BACKWARD else 0
            ops.chirp_mul(x, m0, self.chirp, L, self.local_n, back, 0, 1.0)        # modulate
            self._four_step(m0, m1, m2, FORWARD)
            ops.chirp_mul(m1, m1, self.vhat, L, L, 0, 0, 1.0)                      # convolve
            self._four_step(m1, m0, m2, BACKWARD)
            ops.chirp_mul(m0, w, self.chirp, L, self.local_n, 0, back, 1.0 / self.F)  # demodulate
        self.data, self.work = w, x
        self.norm_exponent += 1
        return 0

    def normalize(self) -> int:
        """(1/sqrt(N))^k, k = executes since the last normalize; the factor in
        single precision for C2C, as the reference's fft1dNormalize."""
        import numpy as np
        if self._state != "planned":
            return ERR_PLAN_NOT_INIT
        k = self.norm_exponent
        if k and self.active:
            if self.precision == C2C:
                f = float(np.float32(1.0) / np.power(np.sqrt(np.float32(self.N)), np.float32(k)))
            else:
                f = 1.0 / math.sqrt(self.N) ** k
            self.ops.scale(self.data, self.L, f)
        self.norm_exponent = 0
        return 0


class CudaOps:
    """Device steps of the distributed transform: kernel-library plans over
    axis subsets, block pack/unpack, scale, and the all-to-all (NCCL for CUDA
    tensors; a gloo group exchanges through host copies)."""

    def __init__(self, precision):
        import torch

        from . import _sm100
        self._sm = _sm100
        self.lib = _sm100.load()
        self.lib.shafft_sm100_plan_create_axes.argtypes = [
            ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.POINTER(ctypes.c_int64),
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        self.lib.shafft_sm100_plan_create_axes_mapped.argtypes = [
            ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.POINTER(ctypes.c_int64),
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
            ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int)]
        self.lib.shafft_sm100_twiddle_rows.argtypes = [
            ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
            ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        for f in (self.lib.shafft_sm100_pack_blocks, self.lib.shafft_sm100_unpack_blocks):
            f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                          ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        self.lib.shafft_sm100_bluestein_chirps.argtypes = [
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
            ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p]
        self.lib.shafft_sm100_chirp_multiply.argtypes = [
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
            ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_void_p]
        self.precision = precision
        self.torch = torch

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def plan(self, dims, axes):
        h = ctypes.c_void_p()
        d = (ctypes.c_int64 * len(dims))(*dims)
        a = (ctypes.c_int * len(axes))(*axes)
        self._sm._check(self.lib.shafft_sm100_plan_create_axes(ctypes.byref(h), len(dims), d,
                                                               self.precision, 0, len(axes), a),
                        "plan_create_axes")
        return h

    def plan_mapped(self, dims, axes, load_map, store_map):
        """Subplan with exchange block maps (outer, n, inner, parts) fused
        into its loads / stores where the library can: (handle, fused bits)."""
        h = ctypes.c_void_p()
        d = (ctypes.c_int64 * len(dims))(*dims)
        a = (ctypes.c_int * len(axes))(*axes)
        lm = None if load_map is None else (ctypes.c_int64 * 4)(*load_map)
        sm = None if store_map is None else (ctypes.c_int64 * 4)(*store_map)
        fused = ctypes.c_int(0)
        self._sm._check(self.lib.shafft_sm100_plan_create_axes_mapped(
            ctypes.byref(h), len(dims), d, self.precision, 0, len(axes), a, lm, sm, ctypes.byref(fused)),
            "plan_create_axes_mapped")
        return h, fused.value

    def destroy(self, h):
        self.lib.shafft_sm100_plan_destroy(h)

    def execute(self, h, src, dst, direction):
        self._sm._check(self.lib.shafft_sm100_execute(h, ctypes.c_void_p(src.data_ptr()),
                                                      ctypes.c_void_p(dst.data_ptr()), int(direction),
                                                      ctypes.c_double(1.0), self._stream()),
                        "execute")

    def pack(self, src, dst, outer, n, inner, P):
        self._sm._check(self.lib.shafft_sm100_pack_blocks(src.data_ptr(), dst.data_ptr(), outer, n, inner,
                                                          P, self.precision, self._stream()), "pack")

    def unpack(self, src, dst, outer, n, inner, P):
        self._sm._check(self.lib.shafft_sm100_unpack_blocks(src.data_ptr(), dst.data_ptr(), outer, n,
                                                            inner, P, self.precision, self._stream()),
                        "unpack")

    def twiddle(self, data, rows, cols, col0, n, sign):
        self._sm._check(self.lib.shafft_sm100_twiddle_rows(data.data_ptr(), rows, cols, col0, n, sign,
                                                           self.precision, self._stream()), "twiddle")

    def scale(self, data, count, factor):
        self._sm._check(self.lib.shafft_sm100_scale(ctypes.c_void_p(data.data_ptr()), count,
                                                    self.precision, ctypes.c_double(factor),
                                                    self._stream()), "scale")

    def empty(self, count):
        dt = self.torch.complex128 if self.precision == Z2Z else self.torch.complex64
        return self.torch.empty(count, dtype=dt, device="cuda")

    def chirps(self, b, v, n, m, n0, m0, count):
        ptr = (lambda t: None if t is None else t.data_ptr())
        self._sm._check(self.lib.shafft_sm100_bluestein_chirps(ptr(b), ptr(v), n, m, n0, m0, count,
                                                               self.precision, self._stream()),
                        "bluestein_chirps")

    def chirp_mul(self, src, dst, factors, count, valid, conj_in, conj_out, scale):
        self._sm._check(self.lib.shafft_sm100_chirp_multiply(src.data_ptr(), dst.data_ptr(),
                                                             factors.data_ptr(), count, valid, conj_in,
                                                             conj_out, scale, self.precision,
                                                             self._stream()), "chirp_multiply")

    def alltoall(self, out, inp, out_counts, in_counts, group, world):
        import torch.distributed as dist
        if world == 1:
            return
        # exchanged as real pairs (2 reals per complex element)
        o = self.torch.view_as_real(out[:sum(out_counts)]).view(-1)
        i = self.torch.view_as_real(inp[:sum(in_counts)]).view(-1)
        oc, ic = [2 * c for c in out_counts], [2 * c for c in in_counts]
        if dist.get_backend(group) == "nccl":
            dist.all_to_all_single(o, i, oc, ic, group=group)
        else:  # host-staged exchange (gloo)
            oh = o.cpu()
            dist.all_to_all_single(oh, i.cpu(), oc, ic, group=group)
            o.copy_(oh)
