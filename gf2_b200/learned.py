"""Learned normalised / offset min-sum: training on the GPU.

The network is the unrolled flooding min-sum decoder with one multiplicative
scale alpha[t, l] and one offset beta[t, l] per unrolled iteration t and row
group l (the 360-row circulant block of DVB-T2 codes):
    c2v = sign * alpha[t, l] * max(min|v2c| - beta[t, l], 0)
It generalises the reference's fixed-weight rules Llr::boxplus_normalized_minsum_n
and Llr::boxplus_offset_minsum_n (crates/gf2-coding/src/llr.rs:352-399).

The unrolled decoder is either the flooding schedule of the reference's
decode_iterative (crates/gf2-coding/src/ldpc/core.rs:889-938) or the layered
schedule (row groups in order, the posterior updated after each); the layered
one converges in about half the iterations, which is what a 10-iteration
decoder of a normal DVB-T2 frame needs.

Training runs entirely on the device: the channel kernel makes the frames
(seeded Philox info bits, encoder, BPSK, AWGN at a per-frame Eb/N0 drawn
uniformly from a range), the library's forward / backward kernels give the
binary cross-entropy of the final soft output and its gradients, and the Adam
kernel updates the weights.  A checkpoint stores the weights, the Adam moments,
the step and the frame counter, so training resumes with identical inputs.

Data parallel training: with a torch.distributed process group of W ranks,
each step's global batch of `batch` frames is split into W contiguous shards
(batch_plan), each rank computes the gradient sums of its shard scaled to the
global mean, and one all-reduce (sum) of the 2 T L gradients and the loss runs
before the Adam step, so every rank applies the same update (NCCL on GPU
ranks).  The frames of a step are the same for every W.
"""
import ctypes

import numpy as np

from . import _capi as C
from .ldpc import LdpcDecoder, awgn_frames, sigma2_from_ebn0, words


_TRAINER_DESTROY = C.lib.gf2c_nms_trainer_destroy


def _vp(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def batch_plan(seed, frame_counter, batch, ebn0_range, rank=0, world=1):
    """Frames of one training step for one rank: (first global frame index,
    frame count, per-frame Eb/N0).  The global batch (frame_counter ..
    frame_counter + batch, Eb/N0 drawn from a generator seeded by (seed,
    frame_counter)) is cut into `world` contiguous shards; rank r takes shard r."""
    rng = np.random.default_rng([seed, frame_counter])
    eb = rng.uniform(ebn0_range[0], ebn0_range[1], batch)
    if batch % world:
        raise ValueError("the global batch must be a multiple of the number of ranks")
    per = batch // world
    lo = rank * per
    return frame_counter + lo, per, eb[lo:lo + per]


def world_info(group=None):
    """(rank, world size) of the process group, (0, 1) without one."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def reduce_gradients(flat, group=None):
    """Sum a tensor holding [gradients..., loss] over the ranks (one all-reduce)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    return flat


def data_parallel_reduce(flat, local_batch, batch, group=None):
    """A shard's [gradients..., loss], each a mean over the shard's frames,
    rescaled to the global batch's mean and summed over the ranks in place."""
    if local_batch != batch:
        flat.mul_(local_batch / batch)
    return reduce_gradients(flat, group)


class NmsTrainer:
    def __init__(self, code, iterations=10, batch=256, ebn0_range=(0.5, 1.5), lr=1e-2, seed=1, device=None,
                 alpha0=0.8, beta0=0.0, betas=(0.9, 0.999), eps=1e-8, schedule=C.SCHED_FLOODING, group=None):
        import torch
        self.torch = torch
        self.code = code
        self.T = int(iterations)
        self.batch = int(batch)  # global batch (all ranks)
        self.schedule = int(schedule)
        self.group = group
        self.rank, self.world = world_info(group)
        if self.batch % self.world:
            raise ValueError("the global batch must be a multiple of the number of ranks")
        self.local_batch = self.batch // self.world
        self.ebn0_range = (float(ebn0_range[0]), float(ebn0_range[1]))
        self.lr = float(lr)
        self.seed = int(seed)
        self.betas = betas
        self.eps = eps
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        h = ctypes.c_void_p()
        C.check(C.lib.gf2c_nms_trainer_create(code.handle, self.T, self.local_batch, ctypes.byref(h)))
        self._h = h
        C.check(C.lib.gf2c_nms_trainer_set_schedule(self._h, self.schedule))
        L = ctypes.c_int32()
        C.check(C.lib.gf2c_nms_trainer_layers(self._h, ctypes.byref(L)))
        self.L = L.value
        # parameters [2, T, L]: alpha then beta (one Adam call for both)
        self.P = torch.empty((2, self.T, self.L), dtype=torch.float32, device=self.device)
        self.P[0].fill_(alpha0)
        self.P[1].fill_(beta0)
        self.G = torch.zeros_like(self.P)
        self.M = torch.zeros_like(self.P)
        self.V = torch.zeros_like(self.P)
        self.loss_buf = torch.zeros(1, dtype=torch.float32, device=self.device)
        self.step_no = 0
        self.frame_counter = 0
        self.history = []

    def __del__(self, _destroy=_TRAINER_DESTROY):  # bound now: module globals may be gone at exit
        h = getattr(self, "_h", None)
        if h:
            _destroy(h)
            self._h = None

    @property
    def alpha(self):
        return self.P[0]

    @property
    def beta(self):
        return self.P[1]

    def loss_grad(self, llr, cw, stream=None):
        """Forward + backward on a device batch; returns (loss tensor [1], grads [2, T, L])."""
        torch = self.torch
        F = llr.shape[0]
        st = stream or torch.cuda.current_stream(self.device)
        C.check(C.lib.gf2c_nms_loss_grad(self._h, _vp(llr), _vp(cw), F, _vp(self.P[0]), _vp(self.P[1]),
                                         _vp(self.G[0]), _vp(self.G[1]), _vp(self.loss_buf), None,
                                         ctypes.c_void_p(st.cuda_stream)))
        return self.loss_buf, self.G

    def make_batch(self):
        """Seeded training frames of this rank for the current frame counter."""
        f0, cnt, eb = batch_plan(self.seed, self.frame_counter, self.batch, self.ebn0_range, self.rank, self.world)
        s2 = np.array([sigma2_from_ebn0(e, self.code.rate()) for e in eb])
        _, cw, llr = awgn_frames(self.code, self.seed, f0, cnt, s2, device=self.device, want_info=False,
                                 want_cw=True)
        return llr, cw

    def train_step(self, sync=True):
        torch = self.torch
        llr, cw = self.make_batch()
        self.loss_grad(llr, cw)
        if self.world > 1:
            # local sums are means over the shard: rescale to the global mean, then sum over ranks
            flat = torch.cat([self.G.reshape(-1), self.loss_buf])
            data_parallel_reduce(flat, self.local_batch, self.batch, self.group)
            self.G.copy_(flat[:-1].view_as(self.G))
            self.loss_buf.copy_(flat[-1:])
        self.step_no += 1
        st = torch.cuda.current_stream(self.device)
        C.check(C.lib.gf2c_adam_step(_vp(self.P), _vp(self.G), _vp(self.M), _vp(self.V), self.P.numel(),
                                     self.lr, self.betas[0], self.betas[1], self.eps, self.step_no,
                                     -4.0, 4.0, ctypes.c_void_p(st.cuda_stream)))
        self.frame_counter += self.batch
        if sync:
            loss = float(self.loss_buf.item())
            self.history.append(loss)
            return loss
        return None

    def train(self, steps, log_every=0, log=print):
        for s in range(steps):
            loss = self.train_step(sync=(log_every and (s % log_every == 0)) or s == steps - 1)
            if log_every and s % log_every == 0 and log:
                log(f"step {self.step_no} frames {self.frame_counter} loss {loss:.5f}")
        return self.history

    def weights(self):
        p = self.P.detach().cpu().numpy()
        return p[0].copy(), p[1].copy()

    def decoder(self, **kw):
        """The inference decoder with the trained weights (same schedule)."""
        a, b = self.weights()
        kw.setdefault("schedule", self.schedule)
        return LdpcDecoder(self.code, algorithm=C.ALGO_NMS, nms_alpha=a, nms_beta=b, **kw)

    # ---- checkpoint / resume ----
    def save(self, path):
        np.savez(path, P=self.P.cpu().numpy(), M=self.M.cpu().numpy(), V=self.V.cpu().numpy(),
                 step=self.step_no, frames=self.frame_counter, seed=self.seed, T=self.T, L=self.L,
                 batch=self.batch, lr=self.lr, ebn0=np.array(self.ebn0_range), history=np.array(self.history),
                 schedule=self.schedule)

    def load(self, path):
        torch = self.torch
        z = np.load(path)
        if int(z["T"]) != self.T or int(z["L"]) != self.L:
            raise ValueError("checkpoint shape does not match this trainer")
        self.P.copy_(torch.from_numpy(z["P"]))
        self.M.copy_(torch.from_numpy(z["M"]))
        self.V.copy_(torch.from_numpy(z["V"]))
        self.step_no = int(z["step"])
        self.frame_counter = int(z["frames"])
        self.seed = int(z["seed"])
        self.history = list(z["history"])
        if "ebn0" in z.files:
            self.ebn0_range = (float(z["ebn0"][0]), float(z["ebn0"][1]))
        return self


def load_weights(path):
    """(alpha, beta) numpy arrays [T, L] of a saved checkpoint."""
    z = np.load(path)
    return z["P"][0].copy(), z["P"][1].copy()
