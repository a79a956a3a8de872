"""The vorticity-confinement adjoint (plume_confinement_adjoint) against the FP64 oracle's confinement operator
(vorticity.py:17-84): for F(u) = u + dt * face_push(u; strength), the adjoint's <J^T a, d> must equal the
directional derivative <a, (F(u + h d) - F(u - h d)) / 2h> taken by central differences of the oracle in
double, and its d/d strength must equal <a, (F(u; s + h) - F(u; s - h)) / 2h>. The identity's share <a, d>
is taken out of both sides, so the comparison is of the confinement's own Jacobian. The velocity is the
operator-test field (smoothed random faces), so the spin and its gradient are nowhere near the push's
|g| < 1e-12 cut-off."""

import numpy as np
import pytest

from oracle import oracle as O
from plume_b200.workloads import operator_fields
from support import ALL_CLOSED, OPEN, oracle_grid

pytestmark = pytest.mark.gpu

DOT_RTOL = 2e-4  # the float32 adjoint's inner products against FP64 central differences (h = 1e-6 of the field)
STRENGTH, DT = 0.3, 0.5


def oracle_confined(fields, cells, cell_m, faces, strength):
    """F(u) on the FP64 oracle: the three face arrays after confinement."""
    o = oracle_grid(cells, cell_m, faces, 1.0, "f64")
    for name in ("u", "v", "w"):
        getattr(o, name).data[...] = fields[name]
    O.VorticityConfinement(o).apply(o, strength, DT)
    return [o.u.data.copy(), o.v.data.copy(), o.w.data.copy()]


def dot(a, b):
    return sum(float(np.sum(x.astype(np.float64) * y.astype(np.float64))) for x, y in zip(a, b))


@pytest.mark.parametrize("cells,faces,cell_m", [((14, 18, 12), OPEN, 0.1), ((9, 11, 7), ALL_CLOSED, 1.0 / 64.0),
                                                ((2, 9, 5), OPEN, 0.05)],
                         ids=["14x18x12-open", "9x11x7-closed", "2x9x5-open"])
def test_confinement_adjoint_is_the_transposed_jacobian(cuda_device, cells, faces, cell_m):
    import torch

    from plume_b200 import _native as N
    from support import cuda_grid

    state = operator_fields(cells, 3, 1.0)
    u = {name: state[name].astype(np.float64) for name in ("u", "v", "w")}
    rng = np.random.default_rng(7)
    a = [rng.normal(size=u[name].shape) for name in ("u", "v", "w")]
    d = [rng.normal(size=u[name].shape) for name in ("u", "v", "w")]

    c = cuda_grid(cells, cell_m, faces, 1.0)
    vel = [torch.from_numpy(np.ascontiguousarray(u[n], dtype=np.float32)).cuda() for n in ("u", "v", "w")]
    adj = [torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda() for x in a]
    scratch = torch.empty(N.lib().plume_confinement_adjoint_scratch_floats(c.info), dtype=torch.float32,
                          device="cuda:0")
    grad_strength = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    N.call("plume_confinement_adjoint", c.info, *(N.ptr(x) for x in vel), *(N.ptr(x) for x in adj), STRENGTH, DT,
           N.ptr(scratch), N.ptr(grad_strength, torch.float64), N.stream())
    a32 = [np.ascontiguousarray(x, dtype=np.float32).astype(np.float64) for x in a]
    jta = [x.cpu().numpy().astype(np.float64) - x0 for x, x0 in zip(adj, a32)]  # the confinement's J^T a

    # the oracle runs from the same float32 velocity values
    base = {n: vel[i].cpu().numpy().astype(np.float64) for i, n in enumerate(("u", "v", "w"))}
    scale = max(float(np.abs(x).max()) for x in base.values())
    h = 1e-6 * scale
    up = oracle_confined({n: base[n] + h * d[i] for i, n in enumerate(("u", "v", "w"))}, cells, cell_m, faces,
                         STRENGTH)
    down = oracle_confined({n: base[n] - h * d[i] for i, n in enumerate(("u", "v", "w"))}, cells, cell_m, faces,
                           STRENGTH)
    directional = dot(a32, [(p - q) / (2.0 * h) for p, q in zip(up, down)]) - dot(a32, d)
    adjoint = dot(jta, d)
    print(f"<a, J d> {directional:.9g}  <J^T a, d> {adjoint:.9g}")
    assert abs(adjoint - directional) <= DOT_RTOL * abs(directional)

    hs = 1e-6
    up = oracle_confined(base, cells, cell_m, faces, STRENGTH + hs)
    down = oracle_confined(base, cells, cell_m, faces, STRENGTH - hs)
    d_strength = dot(a32, [(p - q) / (2.0 * hs) for p, q in zip(up, down)])
    got = float(grad_strength.item())
    print(f"d/d strength: central differences {d_strength:.9g}  adjoint {got:.9g}")
    assert abs(got - d_strength) <= DOT_RTOL * abs(d_strength)

