"""The adjoint kernel (vd_energy_grad_device) wrapped in a torch.autograd.Function.

The wrapper exists only in this test harness.  It differentiates the energy
with respect to the pose's tangent coordinates x = [position (3), rotation
vector w (3), torsions (ntors)], with the pose's quaternion q = exp(w) * q0
(the increment conf.h:367-372 applies).  At w = 0 the adjoint's output is that
derivative exactly: force on the root, torque, dE/dtorsion (tree.h:169-178,
341-348).

Checks, on the adjoint-check workload's ligand shape (40 heavy atoms,
10 torsions) against a 2,000-atom receptor in a 30 A box:
* autograd gradient vs the oracle's FP64 derivative (model.cpp:1324-1333):
  |g - g_ref|_inf <= 1e-3 * max(1, |g_ref|_inf);
* autograd gradient vs central finite differences of the oracle's FP64
  energy with step 1e-4.  The reference's derivative is not the exact
  derivative of its energy: intra pairs take dE/dr from the smooth table's
  own derivative column (precalculate.h:80-95), not the slope of the
  linearly interpolated energy, so torsion derivatives of a 600-pair ligand
  differ from central differences by up to a few tenths.  The test
  therefore requires the GPU gradient to lie as close to the central
  differences as the oracle's derivative does (within 1e-3 * max(1, |g|_inf)),
  and the six rigid-body components, which see few pair terms, to agree
  with the central differences outright (with the cutoff/cell-face caveat
  of the oracle's own finite-difference test: a component may instead agree
  at h = 1e-5 or 1e-6);
* the chain rule through a downstream torch expression.
"""
import numpy as np
import pytest

import oracle_lib as O
from conftest import has_gpu

pytestmark = pytest.mark.gpu

G_TOL = 1e-3


@pytest.fixture(scope="module")
def setup():
    if not has_gpu():
        pytest.skip("needs a CUDA device")
    import torch
    import vdock
    from vdock import synth
    xyz, xs = synth.receptor(2000, 40.0, 4)
    ctx = vdock.Context()
    orc = O.Oracle()
    for o in (ctx, orc):
        o.set_receptor(xyz, xs)
        o.set_box([0.0, 0.0, 0.0], [30.0] * 3)
    lig = synth.ligand(40, 10, 21)
    types = sorted(set(int(t) for t in lig["xs"] if t >= 0))
    ctx.build_grids(types)
    orc.build_grids(types)
    lc, lo = ctx.add_ligand(lig), orc.add_ligand(lig)
    return torch, vdock, ctx, orc, lig, lc, lo


def quat_exp_mul(w, q0, torch):
    """exp(w) * q0 for rotation vectors w [N,3] and unit quaternions q0 [N,4] (w,x,y,z)."""
    ang = torch.linalg.norm(w, dim=1, keepdim=True)
    half = 0.5 * ang
    s = torch.where(ang > 1e-12, torch.sin(half) / torch.clamp(ang, min=1e-12), 0.5 * torch.ones_like(ang))
    a = torch.cat([torch.cos(half), s * w], dim=1)
    aw, ax, ay, az = a.unbind(1)
    bw, bx, by, bz = q0.unbind(1)
    return torch.stack([aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
                        aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw], dim=1)


def make_function(torch, ctx, lig_id):
    class VinaEnergy(torch.autograd.Function):
        @staticmethod
        def forward(fctx, x, q0):
            n, m = x.shape
            pose = torch.cat([x[:, :3], quat_exp_mul(x[:, 3:6], q0, torch), x[:, 6:]], dim=1).contiguous()
            e = torch.empty(n, device=x.device, dtype=torch.float32)
            g = torch.empty(n, m, device=x.device, dtype=torch.float32)
            stream = torch.cuda.current_stream().cuda_stream
            ctx.energy_grad_device(lig_id, n, pose.data_ptr(), e.data_ptr(), g.data_ptr(), stream)
            fctx.save_for_backward(g, x)
            return e

        @staticmethod
        def backward(fctx, ge):
            g, x = fctx.saved_tensors
            assert bool((x[:, 3:6] == 0).all()), "tangent chart: the adjoint is the derivative at w = 0"
            return ge[:, None] * g, None

    return VinaEnergy


def random_inputs(torch, lig, n, seed, nt):
    from vdock import synth
    poses = synth.random_poses(n, nt, -15.0, 15.0, seed=seed)  # uniform in the 30 A box
    x = np.concatenate([poses[:, :3], np.zeros((n, 3), np.float32), poses[:, 7:]], axis=1)
    return poses, torch.tensor(x, device="cuda", requires_grad=True), torch.tensor(poses[:, 3:7], device="cuda")


def test_autograd_matches_oracle_derivative(setup):
    torch, vdock, ctx, orc, lig, lc, lo = setup
    nt = ctx.ntors[lc]
    poses, x, q0 = random_inputs(torch, lig, 128, 31, nt)
    F = make_function(torch, ctx, lc)
    e = F.apply(x, q0)
    w = torch.linspace(0.5, 1.5, len(poses), device="cuda")
    (w * e).sum().backward()  # chain rule through a weighted sum
    g = (x.grad / w[:, None]).cpu().numpy().astype(np.float64)
    e = e.detach().cpu().numpy()
    for i, p in enumerate(poses):
        e_ref, g_ref = orc.eval_deriv(lo, p.astype(np.float64))
        assert abs(e[i] - e_ref) <= 1e-3 + 1e-4 * abs(e_ref), (i, e[i], e_ref)
        assert np.abs(g[i] - g_ref).max() <= G_TOL * max(1.0, np.abs(g_ref).max()), (i, g[i], g_ref)


def quat_increment(q, rot):
    ang = np.linalg.norm(rot)
    if ang < 1e-300:
        return q.copy()
    a = np.concatenate([[np.cos(0.5 * ang)], np.sin(0.5 * ang) * rot / ang])
    r = np.array([a[0] * q[0] - a[1] * q[1] - a[2] * q[2] - a[3] * q[3],
                  a[0] * q[1] + a[1] * q[0] + a[2] * q[3] - a[3] * q[2],
                  a[0] * q[2] - a[1] * q[3] + a[2] * q[0] + a[3] * q[1],
                  a[0] * q[3] + a[1] * q[2] - a[2] * q[1] + a[3] * q[0]])
    return r / np.linalg.norm(r)


def fd_grad(orc, lo, conf, nt, h):
    fd = np.zeros(6 + nt)
    for k in range(6 + nt):
        def shifted(s):
            c = conf.copy()
            if k < 3:
                c[k] += s
            elif k < 6:
                rot = np.zeros(3)
                rot[k - 3] = s
                c[3:7] = quat_increment(c[3:7], rot)
            else:
                c[7 + k - 6] += s
            return orc.eval_deriv(lo, c)[0]
        fd[k] = (shifted(h) - shifted(-h)) / (2 * h)
    return fd


def test_autograd_matches_central_differences(setup):
    torch, vdock, ctx, orc, lig, lc, lo = setup
    nt = ctx.ntors[lc]
    poses, x, q0 = random_inputs(torch, lig, 64, 47, nt)
    _, bmin, bmax = orc.grid_info()
    inside = [i for i, p in enumerate(poses)
              if np.all((lambda c: (c >= bmin) & (c <= bmax))(orc.coords(lo, p.astype(np.float64), lig["n_atoms"])))]
    assert len(inside) >= 4
    F = make_function(torch, ctx, lc)
    F.apply(x, q0).sum().backward()
    g = x.grad.cpu().numpy().astype(np.float64)
    for i in inside[:6]:
        conf = poses[i].astype(np.float64)
        conf[3:7] /= np.linalg.norm(conf[3:7])
        _, g_ref = orc.eval_deriv(lo, conf)
        tol = G_TOL * max(1.0, np.abs(g[i]).max())
        fds = np.stack([fd_grad(orc, lo, conf, nt, h) for h in (1e-4, 1e-5, 1e-6)])
        err_gpu = np.abs(fds[0] - g[i])
        err_ref = np.abs(fds[0] - g_ref)
        assert np.all(err_gpu <= err_ref + tol), (i, (err_gpu - err_ref).max(), tol)
        rigid = np.min(np.abs(fds[:, :6] - g[i][:6]), axis=0)
        assert np.all(rigid <= tol), (i, rigid, tol)


def test_device_entry_points_follow_the_callers_stream(setup):
    """vd_energy_grad_device / vd_energy_device run on the stream they are
    given: work the caller enqueues after them on that stream sees their
    results (here a clone on a side stream), equal bit for bit to the
    host-buffer entry point."""
    torch, vdock, ctx, orc, lig, lc, lo = setup
    from vdock import synth
    nt = ctx.ntors[lc]
    poses = synth.random_poses(4096, nt, -15.0, 15.0, seed=5)
    e_ref, g_ref = ctx.energy_grad(lc, poses)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        dp = torch.from_numpy(poses).cuda()
        de = torch.full((len(poses),), float("nan"), device="cuda")
        dg = torch.full((len(poses), 6 + nt), float("nan"), device="cuda")
        de2 = torch.full((len(poses),), float("nan"), device="cuda")
        ctx.energy_grad_device(lc, len(poses), dp.data_ptr(), de.data_ptr(), dg.data_ptr(), side.cuda_stream)
        ctx.energy_device(lc, len(poses), dp.data_ptr(), de2.data_ptr(), side.cuda_stream)
        e_c, g_c, e2_c = de.clone(), dg.clone(), de2.clone()
    side.synchronize()
    assert np.array_equal(e_c.cpu().numpy(), e_ref) and np.array_equal(g_c.cpu().numpy(), g_ref)
    np.testing.assert_allclose(e2_c.cpu().numpy(), e_ref, rtol=0, atol=1e-5 * np.abs(e_ref).max())
