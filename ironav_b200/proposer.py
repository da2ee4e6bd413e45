"""The learned proposer (the north star's form 4): a small convolutional network that proposes, for each P
macroblock, 4 candidate vectors and logits for its partitioning, which the exact integer cost then judges
(ironav_b200.learned). The network is as specified: 4 conv3x3 layers of 32 channels with ReLU on a 48 x 48
input of two channels (the macroblock's 16 x 16 luma tiled 3 x 3, so every window position meets the current
samples, and the co-located 48 x 48 reference window centred on the macroblock), both u8 / 255, then a linear
head (32 x 48 x 48 = 73,728 features) to 13 outputs: 4 vectors (x, y in units of 32 luma samples, so +-1 spans
+-32) and 5 logits (P_Skip, 16x16, 16x8, 8x16, 8x8). BF16 weights and activations, FP32 accumulation.

Every contraction runs in this library's own tcgen05 kernels (ironav_prop_conv3x3 for the forward pass and the
backward data gradient, ironav_prop_wgrad3x3 for the weight gradients); the input, the head, the loss and Adam
run in its CUDA-core kernels. PyTorch only holds the device buffers and the stream.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .inter import cuda_library

RPIX = 50 * 50  # a sample's padded raster
NOUT = 13
NFEAT = 32 * 48 * 48
MV_SCALE = 128.0  # quarter samples per output unit

SAMPLE_DTYPE = np.dtype([("cur", "<u8"), ("ref", "<u8"), ("w", "<i4"), ("h", "<i4"), ("stride", "<i4"), ("mbx", "<i4"), ("mby", "<i4"),
                         ("ref_stride", "<i4")])
assert SAMPLE_DTYPE.itemsize == 40

# the flat parameter vector: (name, shape)
LAYOUT = [("w1", (9, 32, 16)), ("b1", (32,)), ("w2", (9, 32, 32)), ("b2", (32,)), ("w3", (9, 32, 32)), ("b3", (32,)),
          ("w4", (9, 32, 32)), ("b4", (32,)), ("hw", (NOUT, NFEAT)), ("hb", (NOUT,))]


def _check(status: int, what: str) -> None:
    if status != 0:
        raise RuntimeError(f"{what}: status {status}")


class Proposer:
    """The network's parameters (FP32 masters, BF16 copies for the tensor cores) and Adam state on the device,
    with activation buffers for batches of up to `max_batch` samples."""

    def __init__(self, max_batch: int = 512, seed: int = 0x1A2C, stream=None):
        import torch

        self.torch = torch
        self.lib = cuda_library()
        self.dev = torch.device("cuda", torch.cuda.current_device())
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        sizes = [int(np.prod(s)) for _, s in LAYOUT]
        self.n_params = sum(sizes)
        self.p = torch.zeros(self.n_params, dtype=torch.float32, device=self.dev)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.views, self.gviews = {}, {}
        off = 0
        for (name, shape), n in zip(LAYOUT, sizes):
            self.views[name] = self.p[off:off + n].view(*shape)
            self.gviews[name] = self.g[off:off + n].view(*shape)
            off += n
        self._init(seed)
        bf = torch.bfloat16
        self.wf = {1: torch.zeros((9, 32, 16), dtype=bf, device=self.dev)}
        self.wt = {}
        for l in (2, 3, 4):
            self.wf[l] = torch.zeros((9, 32, 32), dtype=bf, device=self.dev)
            self.wt[l] = torch.zeros((9, 32, 32), dtype=bf, device=self.dev)
        self.hwt = torch.zeros((NFEAT, 16), dtype=torch.float32, device=self.dev)  # the head's packed weights
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.sums = torch.zeros(3, dtype=torch.float32, device=self.dev)
        self.step_count = 0
        self.max_batch = 0
        self.max_grad_batch = 0
        self._alloc(max_batch)
        self.refresh_weights()

    def _init(self, seed: int) -> None:
        torch = self.torch
        g = torch.Generator(device=self.dev).manual_seed(seed)
        with torch.no_grad():
            w1 = torch.randn((9, 32, 16), generator=g, device=self.dev) * np.sqrt(2.0 / (9 * 2))
            w1[:, :, 2:] = 0  # input channels 2..15 carry nothing
            self.views["w1"].copy_(w1)
            for l in (2, 3, 4):
                self.views[f"w{l}"].copy_(torch.randn((9, 32, 32), generator=g, device=self.dev) * np.sqrt(2.0 / (9 * 32)))
            self.views["hw"].copy_(torch.randn((NOUT, NFEAT), generator=g, device=self.dev) * (0.5 / np.sqrt(NFEAT)))

    def _alloc(self, n: int) -> None:
        """The forward pass's buffers for batches of up to n samples."""
        if n <= self.max_batch:
            return
        torch, bf = self.torch, self.torch.bfloat16
        Q = n * RPIX
        self.x0 = torch.zeros((2, Q, 8), dtype=bf, device=self.dev)
        self.z = {l: torch.zeros((4, Q, 8), dtype=bf, device=self.dev) for l in (1, 2, 3, 4)}
        self.out = torch.zeros((n, NOUT), dtype=torch.float32, device=self.dev)
        self.samples_d = torch.zeros(n * SAMPLE_DTYPE.itemsize, dtype=torch.uint8, device=self.dev)
        self.max_batch = n

    def _alloc_grads(self, n: int) -> None:
        """The backward pass's buffers (made on the first training step: inference needs none)."""
        if n <= self.max_grad_batch:
            return
        torch, bf = self.torch, self.torch.bfloat16
        Q = n * RPIX
        self.dz = {l: torch.zeros((4, Q, 8), dtype=bf, device=self.dev) for l in (1, 2, 3, 4)}
        self.dout = torch.zeros((n, NOUT), dtype=torch.float32, device=self.dev)
        self.max_grad_batch = n

    @property
    def _s(self):
        return self.stream.cuda_stream

    def refresh_weights(self) -> None:
        """The BF16 copies of the conv weights (and the data gradient's transposed ones) and the head's packed
        weights, from the masters."""
        lib = self.lib
        _check(lib.ironav_prop_head_pack(self.views["hw"].data_ptr(), self.hwt.data_ptr(), self._s), "head pack")
        _check(lib.ironav_prop_weights(self.views["w1"].data_ptr(), 16, self.wf[1].data_ptr(), None, self._s), "weights 1")
        for l in (2, 3, 4):
            _check(lib.ironav_prop_weights(self.views[f"w{l}"].data_ptr(), 32, self.wf[l].data_ptr(), self.wt[l].data_ptr(), self._s),
                   f"weights {l}")

    def set_samples(self, samples: np.ndarray) -> int:
        """Uploads a batch of samples (SAMPLE_DTYPE) and builds the network's input; returns the batch size."""
        n = len(samples)
        self._alloc(n)
        host = self.torch.from_numpy(np.ascontiguousarray(samples).view(np.uint8))
        with self.torch.cuda.stream(self.stream):
            self.samples_d[: host.numel()].copy_(host, non_blocking=False)
        _check(self.lib.ironav_prop_prep(self.samples_d.data_ptr(), n, self.x0.data_ptr(), self._s), "prep")
        return n

    def set_samples_device(self, d_samples: int, n: int) -> int:
        """Builds the network's input from n samples already in device memory (SAMPLE_DTYPE records)."""
        self._alloc(n)
        _check(self.lib.ironav_prop_prep(d_samples, n, self.x0.data_ptr(), self._s), "prep")
        return n

    def propose(self, n: int, d_cands: int, d_cls: int, min_conf: float = 0.0) -> None:
        """The judge's inputs (ironav_set_learned) from the last forward pass over n macroblocks; a class whose
        probability is below min_conf becomes 5 (unsure: the plain search)."""
        _check(self.lib.ironav_prop_propose(self.out.data_ptr(), n, ctypes.c_float(min_conf), d_cands, d_cls, self._s), "propose")

    def forward(self, n: int, conv_events=None) -> None:
        """Layers 1-4 and the head on the batch set up by set_samples: self.out[:n]. conv_events: a pair of CUDA
        events recorded on the proposer's stream before layer 1 and after layer 4."""
        lib, e = self.lib, self.err.data_ptr()
        if conv_events is not None:
            conv_events[0].record(self.stream)
        _check(lib.ironav_prop_conv3x3(self.x0.data_ptr(), 16, n, self.wf[1].data_ptr(), self.views["b1"].data_ptr(), 1, None,
                                       self.z[1].data_ptr(), e, self._s), "conv 1")
        for l in (2, 3, 4):
            _check(lib.ironav_prop_conv3x3(self.z[l - 1].data_ptr(), 32, n, self.wf[l].data_ptr(), self.views[f"b{l}"].data_ptr(), 1, None,
                                           self.z[l].data_ptr(), e, self._s), f"conv {l}")
        if conv_events is not None:
            conv_events[1].record(self.stream)
        _check(lib.ironav_prop_head_fwd_packed(self.z[4].data_ptr(), n, self.hwt.data_ptr(), self.views["hb"].data_ptr(),
                                               self.out.data_ptr(), self._s), "head")

    def backward(self, n: int, target_mv, target_part) -> None:
        """The loss of the last forward pass against the targets (device tensors: int16 [n, 2] quarter samples,
        uint8 [n]) and every parameter's gradient, accumulated into self.g."""
        lib, e = self.lib, self.err.data_ptr()
        self._alloc_grads(n)
        _check(lib.ironav_prop_loss(self.out.data_ptr(), target_mv.data_ptr(), target_part.data_ptr(), n, self.dout.data_ptr(),
                                    self.sums.data_ptr(), self._s), "loss")
        _check(lib.ironav_prop_head_bwd(self.z[4].data_ptr(), n, self.dout.data_ptr(), self.views["hw"].data_ptr(),
                                        self.gviews["hw"].data_ptr(), self.gviews["hb"].data_ptr(), self.dz[4].data_ptr(), self._s), "head bwd")
        for l in (4, 3, 2):
            _check(lib.ironav_prop_wgrad3x3(self.z[l - 1].data_ptr(), 32, self.dz[l].data_ptr(), n, self.gviews[f"w{l}"].data_ptr(),
                                            self.gviews[f"b{l}"].data_ptr(), e, self._s), f"wgrad {l}")
            _check(lib.ironav_prop_conv3x3(self.dz[l].data_ptr(), 32, n, self.wt[l].data_ptr(), None, 0, self.z[l - 1].data_ptr(),
                                           self.dz[l - 1].data_ptr(), e, self._s), f"dgrad {l}")
        _check(lib.ironav_prop_wgrad3x3(self.x0.data_ptr(), 16, self.dz[1].data_ptr(), n, self.gviews["w1"].data_ptr(),
                                        self.gviews["b1"].data_ptr(), e, self._s), "wgrad 1")

    def update(self, lr: float, lr_head: float | None = None) -> None:
        """Adam on every parameter, then the BF16 copies. The head gets its own step size (lr / 30 by default):
        Adam moves every weight by about its step size, and the head sums 73,728 features, so the conv layers'
        step would move its outputs by tens of units at once."""
        self.step_count += 1
        if lr_head is None:
            lr_head = lr / 30.0
        nconv = self.n_params - NOUT * NFEAT - NOUT
        for off, n, rate in ((0, nconv, lr), (nconv, self.n_params - nconv, lr_head)):
            _check(self.lib.ironav_prop_adam(self.p.data_ptr() + 4 * off, self.g.data_ptr() + 4 * off, self.m.data_ptr() + 4 * off,
                                             self.v.data_ptr() + 4 * off, n, ctypes.c_float(rate), ctypes.c_float(0.9), ctypes.c_float(0.999),
                                             self.step_count, ctypes.c_float(1e-8), self._s), "adam")
        with self.torch.no_grad():
            self.views["w1"][:, :, 2:] = 0
        self.refresh_weights()

    def train_step(self, samples: np.ndarray, target_mv, target_part, lr: float = 1e-3, lr_head: float | None = None) -> None:
        n = self.set_samples(samples)
        self.forward(n)
        self.backward(n, target_mv, target_part)
        self.update(lr, lr_head)

    def check_errors(self) -> None:
        if int(self.err.item()) != 0:
            raise RuntimeError("a tensor-core kernel's wait gave up")

    def state_dict(self) -> dict:
        return {"params": self.p.detach().cpu().numpy().copy(), "step": self.step_count}

    def load_state_dict(self, d: dict) -> None:
        self.p.copy_(self.torch.from_numpy(d["params"]).to(self.dev))
        self.step_count = int(d.get("step", 0))
        self.refresh_weights()
