"""CPU oracle (numpy, FP64) for the learned per-cluster preconditioner.

Test infrastructure only: the tests compare the CUDA path (librepulsor_b200.so,
rpb_mlp_eval / rpb_tpm0_learned_apply / rpb_mlp_train_step) with this restatement.
The learned preconditioner has no counterpart in the reference; its cluster quantities
follow the reference's ClusterTree conventions:

* primitive weights a_i = mean vertex charge * volume and the averaging row a_i/(n+1)
  of the Pre operator (AvOp, src/SimplicialMesh/ComputeNearFarDataOps.hpp:3-63, applied
  by ClusterTree::Pre, src/ClusterTree.hpp:770-857),
* cluster moments as sums over the contiguous primitive range of a cluster
  (src/ClusterTree/ComputeClusterData_Thread.hpp:50-129),
* cluster boxes as the bounding box of the primitives' vertices, radius^2 = |half
  extent|^2 (AABB::FromPrimitives, src/BoundingVolumes/AABB.hpp:160-236),
* the expansion Z_i = sum over the clusters containing i, i.e. PercolateDown followed by
  ClustersToPrimitives (src/ClusterTree/ClusterTreeBase.hpp:452-480,
  src/ClusterTree.hpp:706-768), and the transpose of Pre (Post,
  src/ClusterTree.hpp:860-870).

The MLP reads BF16-rounded weights (round to nearest even) and BF16-rounded layer inputs,
as the device's tensor-core pass does, and is evaluated here in FP64; GPU-vs-oracle
differences come from the FP32 accumulation and from activations that round differently.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

NF, NH, NO = 16, 64, 3
OFF_W1 = 0
OFF_B1 = OFF_W1 + NH * NF
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NO * NH
NPARAM = OFF_B3 + NO
GAIN_CLAMP = 3.0
# level exponent of the multilevel coefficients R_C (A_C / A_root)^k / A_C (kLevelExponent
# in repulsor_b200/csrc/rpb_learned.cu)
LEVEL_EXPONENT = 0.5


def bf16_round(x):
    """float32 -> nearest bfloat16 (ties to even) -> float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(theta, quantize=True):
    w = bf16_round(theta) if quantize else np.asarray(theta, np.float64)
    return (w[OFF_W1:OFF_B1].reshape(NH, NF), w[OFF_B1:OFF_W2], w[OFF_W2:OFF_B2].reshape(NH, NH),
            w[OFF_B2:OFF_W3], w[OFF_W3:OFF_B3].reshape(NO, NH), w[OFF_B3:NPARAM])


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def mlp_forward(theta, F, quantize=True):
    """With quantize (the device's arithmetic): BF16 weights, BF16 layer inputs (features
    and GELU outputs), FP32-or-better accumulation (FP64 here)."""
    W1, b1, W2, b2, W3, b3 = unpack(theta, quantize)
    q = bf16_round if quantize else (lambda x: np.asarray(x, np.float64))
    Fq = q(np.asarray(F, np.float64))
    pre1 = Fq @ W1.T + b1
    h1 = q(gelu(pre1))
    pre2 = h1 @ W2.T + b2
    h2 = q(gelu(pre2))
    O = h2 @ W3.T + b3
    return O, (Fq, pre1, pre2, h1, h2)


def mlp_backward(theta, cache, dO, quantize=True):
    """Gradient of sum(dO * O) with respect to the (BF16-rounded) parameters; the BF16
    rounding of the activations passes gradients straight through."""
    W1, b1, W2, b2, W3, b3 = unpack(theta, quantize)
    F, pre1, pre2, h1, h2 = cache
    g = np.zeros(NPARAM)
    g[OFF_W3:OFF_B3] = (dO.T @ h2).ravel()
    g[OFF_B3:NPARAM] = dO.sum(0)
    d2 = (dO @ W3) * gelu_grad(pre2)
    g[OFF_W2:OFF_B2] = (d2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(0)
    d1 = (d2 @ W2) * gelu_grad(pre1)
    g[OFF_W1:OFF_B1] = (d1.T @ F).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(0)
    return g


class LearnedGeometry:
    """Cluster-tree quantities the learned preconditioner reads, from (V, S) and the tree
    (perm, C_begin, C_end, C_left, C_right) of the mesh."""

    def __init__(self, V, S, tree, charges=None):
        V = np.asarray(V, np.float64)
        S = np.asarray(S, np.int64)
        self.nV = V.shape[0]
        self.dom = S.shape[1] - 1
        perm = np.asarray(tree["perm"], np.int64)
        self.C_begin = np.asarray(tree["C_begin"], np.int64)
        self.C_end = np.asarray(tree["C_end"], np.int64)
        self.C_left = np.asarray(tree["C_left"], np.int64)
        self.C_right = np.asarray(tree["C_right"], np.int64)
        NC = self.C_begin.size
        self.NC = NC
        Sp = S[perm]                                    # simplices in cluster order
        self.Sp = Sp
        H = V[Sp]                                       # N x size x 3
        ch = np.ones(self.nV) if charges is None else np.asarray(charges, np.float64)
        charge = ch[Sp].mean(1)
        if self.dom == 1:
            tau = H[:, 1] - H[:, 0]
            vol = np.linalg.norm(tau, axis=1)
            t = tau / vol[:, None]
        else:
            nu = np.cross(H[:, 1] - H[:, 0], H[:, 2] - H[:, 0])
            ln = np.linalg.norm(nu, axis=1)
            vol = 0.5 * ln
            t = nu / ln[:, None]
        a = charge * vol
        self.a = a
        self.w = a / (self.dom + 1)                     # averaging row of Pre
        cen = H.mean(1)
        # prefix sums -> cluster range sums
        self.A_C = self.range_sums(a[:, None])[:, 0]
        self.c_C = self.range_sums(a[:, None] * cen) / self.A_C[:, None]
        self.an_C = self.range_sums(a[:, None] * t)
        lo = np.array([H[self.C_begin[C]:self.C_end[C]].reshape(-1, 3).min(0) for C in range(NC)])
        hi = np.array([H[self.C_begin[C]:self.C_end[C]].reshape(-1, 3).max(0) for C in range(NC)])
        self.diam = 2.0 * np.sqrt((0.25 * (hi - lo) ** 2).sum(1))
        self.diam = self.diam.astype(np.float32).astype(np.float64)   # stored as float on the device
        depth = np.zeros(NC, np.int64)
        parent = np.full(NC, -1, np.int64)
        for C in range(NC):
            if self.C_left[C] >= 0:
                for X in (self.C_left[C], self.C_right[C]):
                    depth[X] = depth[C] + 1
                    parent[X] = C
        self.depth = depth
        self.parent = parent
        # membership matrix rows: primitive i belongs to every cluster whose range holds i
        leaves = np.where(self.C_left < 0)[0]
        self.leaf_of = np.zeros(len(a), np.int64)
        for C in leaves:
            self.leaf_of[self.C_begin[C]:self.C_end[C]] = C

    def range_sums(self, X):
        P = np.vstack([np.zeros((1, X.shape[1])), np.cumsum(X, 0)])
        return P[self.C_end] - P[self.C_begin]

    def prim_from_vertices(self, R):
        return (self.w[:, None, None] * R[self.Sp]).sum(1)

    def vertices_from_prims(self, Z):
        """Transpose of prim_from_vertices: z_v = sum over the primitives at v of w_i Z_i."""
        z = np.zeros((self.nV, 3))
        for l in range(self.dom + 1):
            np.add.at(z, self.Sp[:, l], self.w[:, None] * Z)
        return z

    def expand(self, O):
        """Z_i = sum over the clusters containing primitive i of O_C."""
        acc = np.zeros((self.NC, O.shape[1]))
        for C in range(self.NC):                        # parents precede children (DFS order)
            p = self.parent[C]
            acc[C] = O[C] + (acc[p] if p >= 0 else 0.0)
        return acc[self.leaf_of]

    def features(self, R):
        s = max(np.sqrt((R * R).sum() / (3 * self.nV)), 1e-300)
        Rc = self.range_sums(self.prim_from_vertices(R))
        NC = self.NC
        F = np.zeros((NC, NF))
        A, c = self.A_C, self.c_C
        dr = max(self.diam[0], 1e-300)
        F[:, 0:3] = Rc / (A[:, None] * s)
        F[:, 3:6] = (c - c[0]) / dr
        F[:, 6:9] = self.an_C / A[:, None]
        F[:, 9] = np.log(A / A[0]) / 10.0
        F[:, 10] = np.log(np.maximum(self.diam, 1e-300) / dr) / 10.0
        F[:, 11] = self.depth / max(self.depth.max(), 1)
        L, Rr = self.C_left, self.C_right
        inner = np.where(L >= 0)[0]
        nrm = np.linalg.norm(Rc, axis=1)
        F[inner, 12] = nrm[L[inner]] / (A[L[inner]] * s)
        F[inner, 13] = nrm[Rr[inner]] / (A[Rr[inner]] * s)
        for col, kid in ((14, L), (15, Rr)):
            for C in inner:
                X = kid[C]
                if L[X] >= 0:
                    F[C, col] = np.linalg.norm(Rc[L[X]] + Rc[Rr[X]]) / (A[X] * s)
        return F.astype(np.float32).astype(np.float64), s

    def apply(self, theta, R, return_cache=False, quantize=True):
        """z = M(R): gains exp(clamp(o_C)) on the multilevel coefficients
        R_C (A_C / A_root)^LEVEL_EXPONENT / A_C, expanded to the primitives, gathered to the
        vertices, column means removed."""
        R = np.asarray(R, np.float64)
        F, s = self.features(R)
        O, cache = mlp_forward(theta, F, quantize)
        O32 = O.astype(np.float32).astype(np.float64) if quantize else O
        gain = np.exp(np.clip(O32, -GAIN_CLAMP, GAIN_CLAMP))
        w = (self.A_C / self.A_C[0]) ** LEVEL_EXPONENT / self.A_C
        Rc = self.range_sums(self.prim_from_vertices(R)) * w[:, None]
        Z = self.expand(gain * Rc)
        z = self.vertices_from_prims(Z)
        z -= z.mean(0)
        if return_cache:
            return z, (cache, O32, gain, Rc)
        return z

    def loss_and_grad(self, theta, R, E, apply_A, quantize=True, reg=0.0):
        """Energy-norm loss 1 - (z.R)^2 / ((z.Az)(E.R)) of z = M(R) and its parameter
        gradient (the gradient includes the gain penalty reg * mean(o^2), the returned loss
        does not); apply_A is the metric product."""
        R = np.asarray(R, np.float64)
        z, (cache, O32, gain, Rc) = self.apply(theta, R, return_cache=True, quantize=quantize)
        Az = apply_A(z)
        zr, zAz, er = (z * R).sum(), (z * Az).sum(), (np.asarray(E) * R).sum()
        loss = 1.0 - zr * zr / (zAz * er)
        g = -2.0 * zr / (zAz * er) * R + 2.0 * zr * zr / (zAz * zAz * er) * Az
        g -= g.mean(0)
        gc = self.range_sums(self.prim_from_vertices(g))
        inside = np.abs(O32) < GAIN_CLAMP
        dO = gc * Rc * gain * inside + 2.0 * reg * O32 / (3.0 * self.NC)
        if quantize:
            dO = dO.astype(np.float32).astype(np.float64)
        return loss, mlp_backward(theta, cache, dO, quantize)

    def apply_frozen(self, theta, R, Y, quantize=True):
        """The application to Y with the gains the network gives for the residual R: the
        linearization of M at R with the gains held fixed (rpb_tpm0_learned_apply_pair)."""
        R = np.asarray(R, np.float64)
        F, s = self.features(R)
        O, _ = mlp_forward(theta, F, quantize)
        O32 = O.astype(np.float32).astype(np.float64) if quantize else O
        gain = np.exp(np.clip(O32, -GAIN_CLAMP, GAIN_CLAMP))
        w = (self.A_C / self.A_C[0]) ** LEVEL_EXPONENT / self.A_C
        Yc = self.range_sums(self.prim_from_vertices(np.asarray(Y, np.float64))) * w[:, None]
        z = self.vertices_from_prims(self.expand(gain * Yc))
        return z - z.mean(0)

    def grad_given(self, theta, R, G, quantize=True, reg=0.0):
        """Objective G . M(R) and its parameter gradient (with the gain penalty
        reg * mean(o^2)) for a given sensitivity G = dL/dz (rpb_mlp_train_step_sens)."""
        R = np.asarray(R, np.float64)
        G = np.asarray(G, np.float64)
        z, (cache, O32, gain, Rc) = self.apply(theta, R, return_cache=True, quantize=quantize)
        g = G - G.mean(0)
        gc = self.range_sums(self.prim_from_vertices(g))
        inside = np.abs(O32) < GAIN_CLAMP
        dO = gc * Rc * gain * inside + 2.0 * reg * O32 / (3.0 * self.NC)
        if quantize:
            dO = dO.astype(np.float32).astype(np.float64)
        return float((G * z).sum()), mlp_backward(theta, cache, dO, quantize)
