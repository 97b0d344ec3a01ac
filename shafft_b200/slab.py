"""Slab-decomposed N-D C2C transform over several GPUs (one process per GPU).

FFTND is the reference's multi-rank FFTND path for one distributed axis
(commDims = [P, 1, ..., 1], src/cpp/slab_nd.cpp:84-254 with nda = 1), built on
torch.distributed for the exchange (NCCL between GPUs) and on the kernel
library for everything on the device:

  forward  local slab [ln0, n1, ..., n_{d-1}] (axis 0 block-partitioned)
           1. transform axes 1..d-1        (shafft_sm100_plan_create_axes)
           2. pack the P column blocks of the last axis (shafft_sm100_pack_blocks)
           3. all-to-all                   (torch.distributed.all_to_all_single)
              -> [n0, n1, ..., ln_{d-1}]   (last axis block-partitioned;
                 blocks arrive as row ranges of axis 0, so no unpack)
           4. transform axis 0
           with TransformLayout INITIAL the exchange is then undone
  backward the same steps in reverse (all-to-all of row ranges, then unpack)

which follows FFTNDPlan::executeImpl (src/cpp/shafft_internal.cpp:62-127):
the same subplan order, the same per-stage layouts (block partition with the
first n % P parts one element longer, detail/partition.hpp:40-44), the same
buffer-swap contract (the result is in the buffer get_buffers() reports as
data) and the (1/sqrt(N))^k normalisation.  Methods return the reference's
status codes.  More than one distributed axis (pencils) returns
ERR_NOT_IMPL.  Ranks beyond prod(commDims) are inactive: they own no data
and take part in the exchanges with empty blocks.  FFT1D (below) is the
reference's distributed 1-D transform (the P x P four-step path).
"""
from __future__ import annotations

import ctypes
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


class SlabLayout:
    """Index bookkeeping of a slab decomposition with one distributed axis:
    stage 0 splits axis 0, stage 1 (after the forward exchange) splits the
    last axis.  Pure host arithmetic."""

    def __init__(self, dims, nparts: int, rank: int):
        self.dims = tuple(int(d) for d in dims)
        self.P = int(nparts)
        self.rank = int(rank)
        self.active = self.rank < self.P
        d = len(self.dims)
        self.mid = math.prod(self.dims[1:-1]) if d > 2 else 1
        self.sub = []
        self.off = []
        for axis in ((0, d - 1) if self.P > 1 else (0,)):
            sub, off = list(self.dims), [0] * d
            if self.P > 1:
                n, s = block_partition(self.dims[axis], self.P, self.rank) if self.active else (0, 0)
                sub[axis], off[axis] = n, s
            self.sub.append(sub)
            self.off.append(off)

    @property
    def nstages(self):
        return len(self.sub)

    def size(self, stage: int) -> int:
        return math.prod(self.sub[stage]) if self.active else 0

    def alloc_size(self) -> int:
        return max(self.size(s) for s in range(self.nstages))

    def axes(self, stage: int):
        """(contiguous axes, distributed axes) of a stage."""
        d = len(self.dims)
        if self.P == 1:
            return list(range(d)), []
        return (list(range(1, d)), [0]) if stage == 0 else (list(range(d - 1)), [d - 1])

    def transform_axes(self, stage: int):
        """Axes the stage's subplan transforms (contiguous and not yet done)."""
        d = len(self.dims)
        if self.P == 1:
            return list(range(d))
        return list(range(1, d)) if stage == 0 else [0]

    def forward_counts(self):
        """(send counts, receive counts) in elements per peer, stage 0 -> 1;
        the backward exchange swaps the two lists."""
        send, recv = [], []
        ln0 = self.sub[0][0]
        for p in range(self.P):
            send.append(ln0 * self.mid * block_partition(self.dims[-1], self.P, p)[0]
                        if self.active else 0)
            recv.append(block_partition(self.dims[0], self.P, p)[0] * self.mid * self.sub[1][-1]
                        if self.active else 0)
        return send, recv


class FFTND:
    """Distributed shafft::FFTND (one distributed axis) over a
    torch.distributed process group; buffers are torch CUDA tensors of at
    least alloc_size() complex elements."""

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
        if nda > 1:
            return ERR_NOT_IMPL  # pencil decompositions (several distributed axes)
        world = dist.get_world_size(group) if dist.is_initialized() else 1
        rank = dist.get_rank(group) if dist.is_initialized() else 0
        if ndim == 1 and world > 1:
            return ERR_INVALID_DECOMP
        P = comm_dims[0]
        if P > world or (nda == 1 and P > dims[-1]):
            return ERR_INVALID_DECOMP
        self.dims, self.precision, self.group = tuple(dims), precision, group
        self.output_policy = output_policy
        self.world, self.rank = world, rank
        self.layout = SlabLayout(dims, P, rank)
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
        self.subplans = []
        if self.layout.active:
            for s in range(self.layout.nstages):
                self.subplans.append(self.ops.plan(self.layout.sub[s], self.layout.transform_axes(s)))
        self.data = self.work = None
        self._state = "planned"
        return 0

    def release(self):
        for p in getattr(self, "subplans", []):
            self.ops.destroy(p)
        self.subplans = []
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
    def _stage_of(self, which):
        if which == TENSOR_LAYOUT_CURRENT:
            return self.stage
        if which == TENSOR_LAYOUT_INITIAL:
            return 0
        if which == TENSOR_LAYOUT_REDISTRIBUTED:
            return self.layout.nstages - 1
        return None

    def get_layout(self, which=TENSOR_LAYOUT_CURRENT):
        s = self._stage_of(which)
        if s is None:
            return ERR_INVALID_LAYOUT, [], []
        return 0, list(self.layout.sub[s]), list(self.layout.off[s])

    def get_axes(self, which=TENSOR_LAYOUT_CURRENT):
        s = self._stage_of(which)
        if s is None:
            return ERR_INVALID_LAYOUT, [], []
        ca, da = self.layout.axes(s)
        return 0, ca, da

    # compute ---------------------------------------------------------------
    def _fft(self, s, direction):
        self.ops.execute(self.subplans[s], self.data, self.work, direction)
        self.data, self.work = self.work, self.data

    def _exchange(self, forward):
        """stage 0 -> 1 (forward) or 1 -> 0; the result is left in data."""
        send, recv = self.layout.forward_counts()
        if not forward:
            send, recv = recv, send
        # ranks beyond the P active ones exchange empty blocks
        pad = [0] * (self.world - len(send))
        send, recv = send + pad, recv + pad
        L = self.layout
        n_last = self.dims[-1]
        if forward:
            if L.active:
                self.ops.pack(self.data, self.work, L.sub[0][0] * L.mid, n_last, L.P)
            self.ops.alltoall(self.data, self.work, recv, send, self.group, self.world)
        else:
            self.ops.alltoall(self.work, self.data, recv, send, self.group, self.world)
            if L.active:
                self.ops.unpack(self.work, self.data, L.sub[0][0] * L.mid, n_last, L.P)
        self.stage = 1 if forward else 0

    def execute(self, direction) -> int:
        if self._state != "planned":
            return ERR_PLAN_NOT_INIT
        if self.layout.active and (self.data is None or self.work is None):
            return ERR_NO_BUFFER
        last = self.layout.nstages - 1
        if direction == FORWARD:
            for s in range(self.layout.nstages):
                if self.layout.active:
                    self._fft(s, FORWARD)
                if s < last:
                    self._exchange(True)
            if self.output_policy == LAYOUT_INITIAL:
                while self.stage > 0:
                    self._exchange(False)
        elif direction == BACKWARD:
            while self.stage < last:  # re-apply the redistribution first
                self._exchange(True)
            for s in range(last, -1, -1):
                if self.layout.active:
                    self._fft(s, BACKWARD)
                if s > 0:
                    self._exchange(False)
        else:
            return ERR_INVALID_STATE
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


class FFT1D:
    """Distributed shafft::FFT1D over a torch.distributed group: the
    reference's P x P four-step path (src/cpp/fft/hipfft_method/1d/
    fft1d_cooley_tukey_executor.hip:175-290), for N divisible by P^2.  Rank r
    holds the contiguous block x[r*L, (r+1)*L), L = N/P, before and after a
    transform.  With C = L/P:

      1. all-to-all of C-element chunks      -> [s][c] = x[s*L + r*C + c]
      2. length-P DFTs over s (one column pass of a [P][C] plan)
                                              -> [k1][c], already the send order
      3. twiddle w_N^{(r*C + c) k1}           (shafft_sm100_twiddle_rows)
      4. all-to-all                           -> [s][c] = column r*... of k1 = r
      5. length-L DFT                         -> X[r + P*k2] at k2
      6. all-to-all of the C-chunks of k2     -> [s][j] = X[r*L + s + P*j]
      7. [P][C] -> [C][P] transpose           (shafft_sm100_unpack_blocks)

    The result is in the buffer get_buffers() reports as data (the buffers
    swap on every execute, Slab1D::swapBuffers).  Lengths not divisible by
    P^2 (the reference's distributed Bluestein) return ERR_NOT_IMPL."""

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
        P = dist.get_world_size(group) if dist.is_initialized() else 1
        r = dist.get_rank(group) if dist.is_initialized() else 0
        if n % (P * P):
            return ERR_NOT_IMPL
        L = n // P
        if local_n != L or local_start != r * L:
            return ERR_INVALID_DECOMP
        self.N, self.P, self.rank, self.L, self.C = n, P, r, L, L // P
        self.precision, self.group, self.ops = precision, group, device_ops
        self._state = "configured"
        return 0

    def plan(self) -> int:
        if self._state == "created":
            return ERR_PLAN_NOT_INIT
        if self._state != "configured":
            return ERR_INVALID_STATE
        if self.ops is None:
            self.ops = CudaOps(self.precision)
        if self.P == 1:
            self.plans = [self.ops.plan([self.N], [0])]
        else:
            self.plans = [self.ops.plan([self.P, self.C], [0]), self.ops.plan([self.L], [0])]
        self.data = self.work = self.scratch = None
        self._state = "planned"
        return 0

    def release(self):
        for h in getattr(self, "plans", []):
            self.ops.destroy(h)
        self.plans = []
        self._state = "released"

    def alloc_size(self) -> int:
        return self.L if self._state in ("configured", "planned") else 0

    def set_buffers(self, data, work) -> int:
        if self._state != "planned":
            return ERR_PLAN_NOT_INIT
        if data is None or work is None:
            return ERR_NULLPTR
        if data.numel() < self.L or work.numel() < self.L or data.data_ptr() == work.data_ptr():
            return ERR_ALLOC
        self.data, self.work = data, work
        self.scratch = data.new_empty(self.L)  # plan-owned, as the reference's dBuf/dTemp
        return 0

    def get_buffers(self):
        return 0, self.data, self.work

    def execute(self, direction) -> int:
        if self._state != "planned":
            return ERR_PLAN_NOT_INIT
        if self.data is None:
            return ERR_NO_BUFFER
        if direction not in (FORWARD, BACKWARD):
            return ERR_INVALID_STATE
        x, w, s = self.data, self.work, self.scratch
        if self.P == 1:
            self.ops.execute(self.plans[0], x, w, direction)
        else:
            P, C, L = self.P, self.C, self.L
            eq = [C] * P
            self.ops.alltoall(w, x, eq, eq, self.group, P)              # 1
            self.ops.execute(self.plans[0], w, s, direction)            # 2  [k1][c]
            self.ops.twiddle(s, P, C, self.rank * C, self.N, -1 if direction == FORWARD else 1)  # 3
            self.ops.alltoall(x, s, eq, eq, self.group, P)              # 4
            self.ops.execute(self.plans[1], x, s, direction)            # 5  X[r + P k2]
            self.ops.alltoall(x, s, eq, eq, self.group, P)              # 6  [s][j]
            self.ops.unpack(x, w, C, P, P)                              # 7  [j][s]
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
        if k:
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
        self.lib.shafft_sm100_twiddle_rows.argtypes = [
            ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
            ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        for f in (self.lib.shafft_sm100_pack_blocks, self.lib.shafft_sm100_unpack_blocks):
            f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                          ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
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

    def destroy(self, h):
        self.lib.shafft_sm100_plan_destroy(h)

    def execute(self, h, src, dst, direction):
        self._sm._check(self.lib.shafft_sm100_execute(h, ctypes.c_void_p(src.data_ptr()),
                                                      ctypes.c_void_p(dst.data_ptr()), int(direction),
                                                      ctypes.c_double(1.0), self._stream()),
                        "execute")

    def pack(self, src, dst, outer, n, P):
        self._sm._check(self.lib.shafft_sm100_pack_blocks(src.data_ptr(), dst.data_ptr(), outer, n, P,
                                                          self.precision, self._stream()), "pack")

    def unpack(self, src, dst, outer, n, P):
        self._sm._check(self.lib.shafft_sm100_unpack_blocks(src.data_ptr(), dst.data_ptr(), outer, n, P,
                                                            self.precision, self._stream()), "unpack")

    def twiddle(self, data, rows, cols, col0, n, sign):
        self._sm._check(self.lib.shafft_sm100_twiddle_rows(data.data_ptr(), rows, cols, col0, n, sign,
                                                           self.precision, self._stream()), "twiddle")

    def scale(self, data, count, factor):
        self._sm._check(self.lib.shafft_sm100_scale(ctypes.c_void_p(data.data_ptr()), count,
                                                    self.precision, ctypes.c_double(factor),
                                                    self._stream()), "scale")

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
