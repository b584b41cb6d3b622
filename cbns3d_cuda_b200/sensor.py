"""The learned shock sensor: data collection, training and inference driver.

All arithmetic runs in the library's kernels (include/cbns_b200.h, "Learned
shock sensor"): faces are sampled with their features and WENO-weight labels
from solver states on the GPU, the network's loss and gradient come from the
hand-written forward/backward kernel, Adam from its update kernel, and
inference from the FP32 or the tcgen05 BF16 forward pass.  torch is used here
only to hold device buffers.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi

NIN, NHID, NPARAM = 15, 32, 1601
# parameter layout: W1[32][15] b1[32] W2[32][32] b2[32] w3[32] b3
P_W1, P_B1, P_W2, P_B2, P_W3, P_B3 = 0, 480, 512, 1536, 1568, 1600


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights, zero biases (FP32)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, dtype=np.float32)
    p[P_W1:P_B1] = rng.uniform(-1, 1, 480) * np.sqrt(6.0 / NIN)
    p[P_W2:P_B2] = rng.uniform(-1, 1, 1024) * np.sqrt(6.0 / NHID)
    p[P_W3:P_B3] = rng.uniform(-1, 1, 32) * np.sqrt(6.0 / NHID)
    return p


def sample_faces(block, which=0, stride=1, offset=0, capacity=None, with_dev=False):
    """Features (n x 15 float32), labels (n uint8) [and deviations, face
    indices] of the sampled faces of a block's state, as torch CUDA tensors."""
    import torch
    IM, JM, KM = block.IM, block.JM, block.KM
    nfaces = (IM - 1) * (JM - 2) * (KM - 2) + (IM - 2) * (JM - 1) * (KM - 2) + (IM - 2) * (JM - 2) * (KM - 1)
    cap = capacity if capacity is not None else (nfaces + stride - 1) // stride
    feat = torch.empty((cap, NIN), dtype=torch.float32, device="cuda")
    lab = torch.empty(cap, dtype=torch.uint8, device="cuda")
    dev = torch.empty(cap, dtype=torch.float32, device="cuda") if with_dev else None
    idx = torch.empty(cap, dtype=torch.int32, device="cuda") if with_dev else None
    cnt = C.c_uint()
    _abi.check(block.lib.cbns_sensor_sample(block.h, which, stride, offset, _ptr(feat), _ptr(lab),
                                            _ptr(dev) if dev is not None else None,
                                            _ptr(idx) if idx is not None else None, cap, C.byref(cnt)),
               "cbns_sensor_sample")
    n = min(cnt.value, cap)
    out = (feat[:n], lab[:n])
    return out + ((dev[:n], idx[:n]) if with_dev else ())


def loss_and_grad(params, X, Y, pos_weight=1.0, stream=None):
    import torch
    lib = _abi.load()
    g = torch.empty(NPARAM, dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    _abi.check(lib.cbns_mlp_grad(_ptr(params), _ptr(X), _ptr(Y), X.shape[0], float(pos_weight), _ptr(g), _ptr(loss),
                                 C.c_void_p(stream or 0)), "cbns_mlp_grad")
    return loss, g


def predict(params, X, tensor_cores=False):
    import torch
    lib = _abi.load()
    out = torch.empty(X.shape[0], dtype=torch.float32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    _abi.check(lib.cbns_mlp_predict(_ptr(params), _ptr(X), X.shape[0], _ptr(out), int(tensor_cores), _ptr(status),
                                    None), "cbns_mlp_predict")
    torch.cuda.synchronize()
    if int(status.item()) != 0:
        raise RuntimeError("tensor-core inference timed out waiting for the MMA")
    return out


def train(X, Y, epochs=3, batch=16384, lr=3e-3, pos_weight=None, seed=0, params=None, log=None, cosine=False):
    """Adam on the weighted cross-entropy; returns (params tensor, loss history).
    cosine: decay the learning rate to 0 over the run (half a cosine)."""
    import torch
    lib = _abi.load()
    n = X.shape[0]
    if pos_weight is None:
        pos = float(Y.float().mean().item())
        pos_weight = min(50.0, (1.0 - pos) / max(pos, 1e-6)) if pos > 0 else 1.0
    P = torch.from_numpy(init_params(seed) if params is None else np.asarray(params, np.float32)).cuda()
    M = torch.zeros_like(P)
    V = torch.zeros_like(P)
    G = torch.empty_like(P)
    L = torch.empty(1, dtype=torch.float32, device="cuda")
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    step = 0
    hist = []
    total = epochs * ((n + batch - 1) // batch)
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=gen)
        tot = 0.0
        nb = 0
        for b0 in range(0, n, batch):
            idx = perm[b0:b0 + batch]
            xb = X[idx].contiguous()
            yb = Y[idx].contiguous()
            _abi.check(lib.cbns_mlp_grad(_ptr(P), _ptr(xb), _ptr(yb), xb.shape[0], float(pos_weight), _ptr(G),
                                         _ptr(L), None), "cbns_mlp_grad")
            lr_now = lr * 0.5 * (1.0 + np.cos(np.pi * step / total)) if cosine else lr
            step += 1
            _abi.check(lib.cbns_mlp_adam(_ptr(P), _ptr(G), _ptr(M), _ptr(V), step, float(lr_now), None),
                       "cbns_mlp_adam")
            if nb % 16 == 0:
                tot += float(L.item())
            nb += 1
        hist.append(tot / max(1, (nb + 15) // 16))
        if log:
            log(f"epoch {ep}: loss {hist[-1]:.5f}")
    return P, hist


def save_weights_bin(path, params, tau):
    """The weights file cbns_sensor_load_file reads: "CBNSSNS1", uint32 1601,
    float32 tau, 1601 float32 parameters (little endian)."""
    import struct
    p = np.ascontiguousarray(params, dtype="<f4").reshape(-1)
    assert p.size == NPARAM
    with open(path, "wb") as f:
        f.write(b"CBNSSNS1" + struct.pack("<If", NPARAM, float(tau)) + p.tobytes())
