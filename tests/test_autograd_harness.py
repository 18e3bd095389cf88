"""CPU check of the torch.autograd harness (tests/gatt_autograd.py) itself, with a stand-in
solver whose Jacobians are known in closed form: the wrappers must hand torch the vjp and jvp
the entry points return, in the flat U, V, W, R, E layout.  The GPU tests then use the same
wrappers on the real entry points."""
import numpy as np
import torch
import torch.autograd.forward_ad as fwAD

from gatt_autograd import RHS, Steps

KEYS = ("U", "V", "W", "R", "E")


class FakeSolver:
    """F(q) = q * q + sin(R) on every field; the run maps q to a fixed linear map M q per step."""

    def __init__(self, n, seed=0):
        self.n = n
        rng = np.random.default_rng(seed)
        self.M = np.eye(5 * n) + 0.05 * rng.standard_normal((5 * n, 5 * n))
        self.state = None

    def _pack(self, f):
        return np.concatenate([np.asarray(f[k], dtype=np.float64).ravel() for k in KEYS])

    def _unpack(self, v):
        return {k: v[i * self.n:(i + 1) * self.n].copy() for i, k in enumerate(KEYS)}

    def nseq(self, f):
        return {k: f[k] * f[k] + np.sin(f["R"]) for k in KEYS}

    def rhs_jvp(self, q, dq):
        return {k: 2 * q[k] * dq[k] + np.cos(q["R"]) * dq["R"] for k in KEYS}

    def rhs_vjp(self, q, a):
        out = {k: 2 * q[k] * a[k] for k in KEYS}
        out["R"] = out["R"] + np.cos(q["R"]) * sum(a[k] for k in KEYS)
        return out

    def upload(self, f):
        self.state = self._pack(f)

    def run(self, nsteps, t0, dt):
        for _ in range(nsteps):
            self.state = self.M @ self.state + 0.01 * self.state ** 2

    def download(self):
        return self._unpack(self.state)

    def jvp(self, dq, nsteps, t0, dt):
        x, v = self.state.copy(), self._pack(dq)
        for _ in range(nsteps):
            v = self.M @ v + 0.02 * x * v
            x = self.M @ x + 0.01 * x ** 2
        self.state = x
        return self._unpack(v)

    def vjp(self, lam, nsteps, t0, dt, checkpoint_every=1):
        xs = [self.state.copy()]
        for _ in range(nsteps):
            xs.append(self.M @ xs[-1] + 0.01 * xs[-1] ** 2)
        lv = self._pack(lam)
        for s in range(nsteps - 1, -1, -1):
            lv = self.M.T @ lv + 0.02 * xs[s] * lv
        return self._unpack(lv)


def test_harness_rhs_and_steps_pass_gradcheck():
    g = FakeSolver(6)
    q = torch.from_numpy(np.random.default_rng(1).uniform(0.5, 1.5, 30)).requires_grad_(True)
    assert torch.autograd.gradcheck(lambda x: RHS.apply(x, g), (q,), check_forward_ad=True,
                                    check_undefined_grad=False)
    assert torch.autograd.gradcheck(lambda x: Steps.apply(x, g, 3, 0.0, 0.1, 1), (q,), check_forward_ad=True,
                                    check_undefined_grad=False)


def test_harness_dot_product():
    g = FakeSolver(6, seed=2)
    rng = np.random.default_rng(3)
    q0 = torch.from_numpy(rng.uniform(0.5, 1.5, 30))
    v, w = torch.from_numpy(rng.standard_normal(30)), torch.from_numpy(rng.standard_normal(30))
    with fwAD.dual_level():
        jv = fwAD.unpack_dual(Steps.apply(fwAD.make_dual(q0, v), g, 4, 0.0, 0.1, 2)).tangent
    q = q0.clone().requires_grad_(True)
    (jtw,) = torch.autograd.grad(Steps.apply(q, g, 4, 0.0, 0.1, 2), q, w)
    assert abs(float(torch.dot(jv, w) - torch.dot(v, jtw))) < 1e-12 * abs(float(torch.dot(jv, w)))
