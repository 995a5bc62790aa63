"""Numpy restatement of one rank of the decomposed BiCGStab (TEST
INFRASTRUCTURE: it stands in for the library's hicarw_dist_* primitives where
no GPU is present, so that the host-side schedule of hicar_b200.decomp runs on
gloo ranks in the CPU test suite).

It follows wind_iterative.F90 at one rank of a decomposition: the probed
15-point operator (spmv :883-907) on the rank's block with a one-cell ring
(identity rows on the physical boundary and the ghost planes; halo cells on
the rank-edge sides, which are not rows of this rank), the Jacobi-Richardson
preconditioner with a zero halo (apply_precond :1268-1315), the BiCGStab
recurrences and stopping tests (:555-791) with local dot products that the
caller sums over ranks.  Arrays: (ny+2, nz+2, nx+2) FP64, coefficients
(15, ny, nz, nx) in the order A..O.
"""
import numpy as np
import torch

# offsets (dk, dj, di) of the coefficients A..O (the probed operator's slots)
OFF = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 0, 1), (0, 0, -1), (0, 1, 0), (0, -1, 0), (1, 0, 1), (1, 0, -1),
       (-1, 0, 1), (-1, 0, -1), (1, 1, 0), (1, -1, 0), (-1, 1, 0), (-1, -1, 0)]
# spmv's term order (:883-907): O G M K C J E A D I B H N F L
ORDER = [14, 6, 12, 10, 2, 9, 4, 0, 3, 8, 1, 7, 13, 5, 11]
BREAKDOWN = 1.0e-30


class NumpyRank:
    def __init__(self, coefs, edges: int, tol_rel=1e-5, tol_abs=1e-10, max_iters=1500, sweeps=2):
        self.c = np.asarray(coefs, np.float64)
        _, ny, nz, nx = self.c.shape
        self.nx, self.ny, self.nz = nx, ny, nz
        self.edges = edges
        self.tol_rel, self.tol_abs, self.max_iters, self.sweeps = tol_rel, tol_abs, max_iters, sweeps
        shape = (ny + 2, nz + 2, nx + 2)
        self.owned = np.ones(shape, bool)  # rows of this rank
        if edges & 1:
            self.owned[:, :, 0] = False
        if edges & 2:
            self.owned[:, :, -1] = False
        if edges & 4:
            self.owned[0] = False
        if edges & 8:
            self.owned[-1] = False
        self.dinv = np.ones(shape)
        self.dinv[1:-1, 1:-1, 1:-1] = 1.0 / self.c[0]
        self.dinv[~self.owned] = 0.0  # the preconditioner's zero halo
        z = np.zeros(shape)
        self.x, self.r, self.rhat, self.p, self.phat, self.v, self.s, self.shat, self.t = (z.copy() for _ in range(9))
        self.st = {}

    def op(self, x):
        y = x.copy()  # identity rows (ring, ghost planes); halo rows are not used
        acc = np.zeros((self.ny, self.nz, self.nx))
        for q in ORDER:
            dk, dj, di = OFF[q]
            acc = acc + self.c[q] * x[1 + dj:self.ny + 1 + dj, 1 + dk:self.nz + 1 + dk, 1 + di:self.nx + 1 + di]
        y[1:-1, 1:-1, 1:-1] = acc
        return y

    def dot(self, a, b):
        return float(np.sum((a * b)[self.owned]))

    def _m(self, x):
        y = self.dinv * x
        for _ in range(2, self.sweeps + 1):
            y = y + self.dinv * (x - self.op(y))
        return y

    # ---- the primitives of hicar_b200.decomp.rank_schedule ----
    def setup(self, rhs):
        self.b = np.asarray(rhs, np.float64)
        self.r = self.b - self.op(self.x)
        self.rhat, self.p = self.r.copy(), self.r.copy()
        return torch.tensor([self.dot(self.rhat, self.r), self.dot(self.r, self.r), self.dot(self.b, self.b)],
                            dtype=torch.float64)

    def apply(self, kind, tot):
        t = [float(v) for v in tot]
        st = self.st
        if kind == 0:
            rn = np.sqrt(t[1])
            st.update(rho=t[0], rnorm=rn, res0=rn, target=max(self.tol_abs, self.tol_rel * np.sqrt(t[2])), it=0,
                      stop=0, status=1, alpha=1.0, omega=1.0, upd_r=0, upd_p=0)
            if rn <= st["target"]:
                st.update(status=0, stop=1)
        elif kind == 1:
            if st["stop"]:
                return
            st["it"] += 1
            if abs(t[0]) < BREAKDOWN:
                st.update(status=2, stop=1)
            else:
                st["alpha"] = st["rho"] / t[0]
        else:
            if st["stop"]:
                return
            ts, tt, rs, rt, ss = t
            st.update(upd_r=0, upd_p=0)
            if tt < BREAKDOWN:
                st.update(status=2, stop=1)
                return
            w = ts / tt
            rho_new = rs - w * rt
            rn = np.sqrt(max(ss - 2.0 * w * ts + w * w * tt, 0.0))
            st.update(omega=w, rnorm=rn)
            if rn <= st["target"]:
                st.update(status=0, stop=1)
                return
            if abs(w) < BREAKDOWN:
                st.update(status=2, stop=1)
                return
            st["upd_r"] = 1
            if abs(st["rho"]) < BREAKDOWN:
                st.update(status=2, stop=1)
                return
            st["beta"] = (rho_new / st["rho"]) * (st["alpha"] / w)
            st["upd_p"] = 1
            st["rho"] = rho_new
            if st["it"] >= self.max_iters:
                st.update(status=1, stop=1)

    def precond(self, which):
        if which == 0:
            self.phat = self._m(self.p)
        else:
            self.s = self.r - self.st["alpha"] * self.v
            self.shat = self._m(self.s)

    def face_buffer(self, side):
        return torch.zeros((self.ny + 2, self.nz + 2) if side < 2 else (self.nz + 2, self.nx + 2), dtype=torch.float64)

    def face(self, vec, side, unpack, buf=None):
        a = self.phat if vec == 0 else self.shat
        sel = {0: (slice(None), slice(None), 0 if unpack else 1),
               1: (slice(None), slice(None), -1 if unpack else -2),
               2: (0 if unpack else 1, slice(None), slice(None)),
               3: (-1 if unpack else -2, slice(None), slice(None))}[side]
        if unpack:
            a[sel] = buf.numpy()
            return buf
        out = self.face_buffer(side)
        out.copy_(torch.from_numpy(np.ascontiguousarray(a[sel])))
        return out

    def spmv(self, which):
        if which == 0:
            self.v = self.op(self.phat)
            return torch.tensor([self.dot(self.rhat, self.v)], dtype=torch.float64)
        self.t = self.op(self.shat)
        return torch.tensor([self.dot(self.t, self.s), self.dot(self.t, self.t), self.dot(self.rhat, self.s),
                             self.dot(self.rhat, self.t), self.dot(self.s, self.s)], dtype=torch.float64)

    def update(self):
        st = self.st
        if st.get("halted"):
            return
        self.x = self.x + st["alpha"] * self.phat + st["omega"] * self.shat
        if st["upd_r"]:
            self.r = self.s - st["omega"] * self.t
            if st["upd_p"]:
                self.p = self.r + st["beta"] * (self.p - st["omega"] * self.v)
        if st["stop"]:
            st["halted"] = True

    def stopped(self):
        return bool(self.st["stop"])

    def stats(self):
        return {"status": self.st["status"], "iterations": self.st["it"], "res_final": self.st["rnorm"]}

    def lam(self):
        return self.x
