"""Adam optimizer over the native kernels, interface-compatible with
``svraster_cuda.sparse_adam.SparseAdam`` (backends/cuda/svraster_cuda/sparse_adam.py:13-72).

``sparse=True`` skips elements whose gradient is exactly zero (their moments
are left untouched), ``biased=True`` drops the bias correction.
:class:`FusedSparseAdam` updates every parameter group in one launch.
"""
import ctypes

import torch

from . import _C
from ._native import check, lib


class SparseAdam(torch.optim.Optimizer):

    def __init__(self, params, lr=1e-3, betas=(0.9, 0.999), eps=1e-15, biased=False, sparse=False):
        if not 0.0 <= lr:
            raise ValueError("Invalid learning rate: {}".format(lr))
        if not 0.0 <= eps:
            raise ValueError("Invalid epsilon value: {}".format(eps))
        if not 0.0 <= betas[0] < 1.0:
            raise ValueError("Invalid beta parameter at index 0: {}".format(betas[0]))
        if not 0.0 <= betas[1] < 1.0:
            raise ValueError("Invalid beta parameter at index 1: {}".format(betas[1]))
        super().__init__(params, dict(lr=lr, betas=betas, eps=eps))
        self.biased = biased
        self.sparse = sparse

    def _state(self, p):
        st = self.state[p]
        if len(st) == 0:
            st['step'] = 0
            st['exp_avg'] = torch.zeros_like(p, memory_format=torch.preserve_format)
            st['exp_avg_sq'] = torch.zeros_like(p, memory_format=torch.preserve_format)
        return st

    @torch.no_grad()
    def step(self):
        for group in self.param_groups:
            lr = group['lr']
            beta1, beta2 = group['betas']
            eps = group['eps']
            for p in group['params']:
                if p.grad is None:
                    continue
                st = self._state(p)
                st['step'] += 1
                if self.biased:
                    _C.biased_adam_step(self.sparse, p, p.grad, st['exp_avg'], st['exp_avg_sq'], lr, beta1, beta2,
                                        eps)
                else:
                    _C.unbiased_adam_step(self.sparse, p, p.grad, st['exp_avg'], st['exp_avg_sq'], st['step'], lr,
                                          beta1, beta2, eps)


class FusedSparseAdam(SparseAdam):
    """Unbiased Adam with every parameter updated in a single kernel launch.

    Same per-element arithmetic as ``SparseAdam(biased=False)``; parameters may
    be fp32 or bf16 (moments stay fp32).  All groups must share ``betas`` and
    ``eps``.
    """

    @torch.no_grad()
    def step(self):
        if self.biased:
            raise ValueError("FusedSparseAdam implements the unbiased update only")
        items = []
        betas = eps = None
        for group in self.param_groups:
            if betas is None:
                betas, eps = group['betas'], group['eps']
            elif tuple(group['betas']) != tuple(betas) or group['eps'] != eps:
                raise ValueError("FusedSparseAdam needs identical betas/eps across groups")
            for p in group['params']:
                if p.grad is None:
                    continue
                st = self._state(p)
                st['step'] += 1
                if st['exp_avg'].dtype != torch.float32:
                    st['exp_avg'] = st['exp_avg'].float()
                    st['exp_avg_sq'] = st['exp_avg_sq'].float()
                items.append((p, p.grad, st, group['lr']))
        for i in range(0, len(items), 8):
            chunk = items[i:i + 8]
            n = len(chunk)
            dev = chunk[0][0].device
            for p, g, st, _ in chunk:
                if p.dtype not in (torch.float32, torch.bfloat16) or g.dtype != torch.float32:
                    raise RuntimeError("FusedSparseAdam: params fp32/bf16, grads fp32")
                if not (p.is_contiguous() and g.is_contiguous()):
                    raise RuntimeError("FusedSparseAdam: contiguous params and grads required")
            P = (ctypes.c_void_p * n)(*[c[0].data_ptr() for c in chunk])
            B = (ctypes.c_int * n)(*[int(c[0].dtype == torch.bfloat16) for c in chunk])
            G = (ctypes.c_void_p * n)(*[c[1].data_ptr() for c in chunk])
            M = (ctypes.c_void_p * n)(*[c[2]['exp_avg'].data_ptr() for c in chunk])
            V = (ctypes.c_void_p * n)(*[c[2]['exp_avg_sq'].data_ptr() for c in chunk])
            Nn = (ctypes.c_int64 * n)(*[c[0].numel() for c in chunk])
            S = (ctypes.c_double * n)(*[float(c[2]['step']) for c in chunk])
            LR = (ctypes.c_double * n)(*[float(c[3]) for c in chunk])
            with torch.cuda.device(dev):
                st = lib().svr_fused_adam_step(n, int(bool(self.sparse)), P, B, G, M, V, Nn, S, LR,
                                               float(betas[0]), float(betas[1]), float(eps),
                                               ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
            check(st, "fused_adam_step")
