"""6-DOF pose refinement by L-BFGS on the masked normalised CC, driven through the C-ABI
forward + adjoint (emc_cc_adjoint_batch).

It replaces the fine local angular grid of the alignment loop (the refinement grid around the
coarse best, alignment/BH_alignRaw3d_v2.m:1448-1641) by gradient ascent from the coarse-search
result: every particle keeps its own L-BFGS state, and all particles advance in lockstep so that
each objective evaluation is a single batched launch over every particle still running.

Pose vector: (phi, theta, psi) in degrees and (tx, ty, tz) in voxels, relative to the particle's
prior rotation R_prior (RotMat = R_prior * defineMatrix([phi, theta, psi - phi], 'inv')); the shift
is applied in real space with the reference sampling ('forward' semantics).
"""
import ctypes as C

import numpy as np
import torch

from . import _lib as L


class BatchObjective:
    """-CC and its gradient for many (particle, pose) items in one launch."""

    def __init__(self, search, ref_ids, templates, energies, priors, interp="linear"):
        self.s = search
        self.n = len(ref_ids)
        self.ref_ids = np.ascontiguousarray(ref_ids, dtype=np.int32)
        self.keep = list(templates)
        self.h_ptrs = (C.c_void_p * self.n)(*[t.data_ptr() for t in templates])
        self.energies = np.ascontiguousarray(energies, dtype=np.float64)
        self.priors = np.ascontiguousarray(
            np.stack([np.asarray(p, dtype=np.float64).reshape(3, 3).flatten(order="F") for p in priors]))
        self.interp = {"linear": L.INTERP_LINEAR, "cubic": L.INTERP_CUBIC}[interp]
        self.evals = 0

    def __call__(self, poses, idx=None):
        """poses: (k, 6) for the items idx (all items when None).  Returns (-cc, -grad)."""
        f, g = self.cc_grad(poses, idx)
        return -f, -g

    def cc_grad(self, poses, idx=None):
        """poses: (k, 6) for the items idx (all items when None).  Returns (cc, dcc/dpose)."""
        idx = np.arange(self.n) if idx is None else np.asarray(idx)
        k = len(idx)
        poses = np.ascontiguousarray(poses, dtype=np.float64).reshape(k, 6)
        ids = np.ascontiguousarray(self.ref_ids[idx])
        hp = (C.c_void_p * k)(*[self.h_ptrs[i] for i in idx])
        en = np.ascontiguousarray(self.energies[idx])
        pr = np.ascontiguousarray(self.priors[idx])
        cc = np.zeros(k)
        g = np.zeros((k, 6))
        pd = C.POINTER(C.c_double)
        L.call("emc_cc_adjoint_batch", self.s._h, k, ids.ctypes.data_as(C.POINTER(C.c_int)), hp,
               en.ctypes.data_as(pd), pr.ctypes.data_as(pd), poses.ctypes.data_as(pd), self.interp,
               cc.ctypes.data_as(pd), g.ctypes.data_as(pd), C.c_void_p(torch.cuda.current_stream().cuda_stream))
        self.evals += k
        return cc, g


class CCPose(torch.autograd.Function):
    """torch.autograd.Function over the forward + adjoint (emc_cc_adjoint_batch).
    ``CCPose.apply(poses, objective)`` maps a (k, 6) float64 tensor of poses (phi, theta, psi in
    degrees; tx, ty, tz in voxels) to the k masked normalised CCs of a BatchObjective; backward
    returns grad_out * dCC/dpose from the same launch (the adjoint kernel evaluates the value and its
    exact gradient together, so nothing is recomputed).  For tests and for optimisers written against
    torch; the L-BFGS below calls the objective directly."""

    @staticmethod
    def forward(ctx, poses, objective):
        cc, g = objective.cc_grad(poses.detach().cpu().numpy())
        ctx.save_for_backward(torch.from_numpy(g).to(poses))
        return torch.from_numpy(cc).to(poses)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out.unsqueeze(-1) * g, None


def lbfgs(objective, x0, n_iter=20, memory=6, max_ls=8, c1=1e-4, first_step=1.0, tol=1e-10):
    """Minimises objective (batched over items) from x0 (k, d) with per-item L-BFGS and a
    backtracking Armijo line search.  Returns (x, f, history of f per iteration)."""
    x = np.array(x0, dtype=np.float64)
    k, d = x.shape
    f, g = objective(x)
    S = np.zeros((k, memory, d))
    Y = np.zeros((k, memory, d))
    rho = np.zeros((k, memory))
    used = np.zeros(k, dtype=int)
    head = np.zeros(k, dtype=int)
    active = np.ones(k, dtype=bool)
    hist = [f.copy()]
    for it in range(n_iter):
        act = np.nonzero(active)[0]
        if len(act) == 0:
            break
        # two-loop recursion, vectorised over the active items
        q = g[act].copy()
        alpha = np.zeros((len(act), memory))
        for j in range(memory):
            slot = (head[act] - 1 - j) % memory
            ok = j < used[act]
            s_j = S[act, slot]
            y_j = Y[act, slot]
            a = np.where(ok, rho[act, slot] * np.einsum("ij,ij->i", s_j, q), 0.0)
            alpha[:, j] = a
            q -= a[:, None] * y_j
        last = (head[act] - 1) % memory
        sy = np.einsum("ij,ij->i", S[act, last], Y[act, last])
        yy = np.einsum("ij,ij->i", Y[act, last], Y[act, last])
        gamma = np.where(used[act] > 0, sy / np.maximum(yy, 1e-300), 0.0)
        first = used[act] == 0
        gnorm = np.abs(g[act]).max(axis=1)
        gamma = np.where(first, first_step / np.maximum(gnorm, 1e-300), gamma)
        r = gamma[:, None] * q
        for j in reversed(range(memory)):
            slot = (head[act] - 1 - j) % memory
            ok = j < used[act]
            b = np.where(ok, rho[act, slot] * np.einsum("ij,ij->i", Y[act, slot], r), 0.0)
            r += (alpha[:, j] - b)[:, None] * S[act, slot]
        direction = -r
        slope = np.einsum("ij,ij->i", g[act], direction)
        bad = slope >= 0
        direction[bad] = -g[act][bad] * (first_step / np.maximum(gnorm[bad], 1e-300))[:, None]
        slope[bad] = np.einsum("ij,ij->i", g[act][bad], direction[bad])
        # backtracking line search, all items in lockstep
        step = np.ones(len(act))
        done = np.zeros(len(act), dtype=bool)
        f_new = f[act].copy()
        g_new = g[act].copy()
        x_new = x[act].copy()
        for _ in range(max_ls):
            todo = np.nonzero(~done)[0]
            if len(todo) == 0:
                break
            xt = x[act][todo] + step[todo, None] * direction[todo]
            ft, gt = objective(xt, act[todo])
            accept = ft <= f[act][todo] + c1 * step[todo] * slope[todo]
            acc_i = todo[accept]
            f_new[acc_i], g_new[acc_i], x_new[acc_i] = ft[accept], gt[accept], xt[accept]
            done[acc_i] = True
            step[todo[~accept]] *= 0.5
        # update histories of the items that moved
        moved = act[done]
        s_vec = x_new[done] - x[moved]
        y_vec = g_new[done] - g[moved]
        sy = np.einsum("ij,ij->i", s_vec, y_vec)
        good = sy > 1e-12
        mg = moved[good]
        S[mg, head[mg]] = s_vec[good]
        Y[mg, head[mg]] = y_vec[good]
        rho[mg, head[mg]] = 1.0 / sy[good]
        head[mg] = (head[mg] + 1) % memory
        used[mg] = np.minimum(used[mg] + 1, memory)
        improvement = f[moved] - f_new[done]
        x[moved], f[moved], g[moved] = x_new[done], f_new[done], g_new[done]
        # items whose line search failed or stalled stop
        active[act[~done]] = False
        active[moved[improvement < tol]] = False
        hist.append(f.copy())
    return x, f, hist


def geodesic_deg(Ra, Rb):
    """Angle of Ra^T Rb in degrees (rotation distance)."""
    c = (np.trace(np.swapaxes(Ra, -1, -2) @ Rb, axis1=-2, axis2=-1) - 1.0) / 2.0
    return np.degrees(np.arccos(np.clip(c, -1.0, 1.0)))
