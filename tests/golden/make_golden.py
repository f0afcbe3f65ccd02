"""Generate the golden fixtures in this directory by running the reference.

Run where a torch-admp checkout is available (it imports the reference):
``TORCH_ADMP_REFERENCE=<checkout> python tests/golden/make_golden.py [case ...]``.

Each ``*.npz`` holds the inputs of one case together with what the
reference's own FP64 CPU path (torch-admp 1.1.5, imported through
``_ref_import``) returns for them: energies, energy components and the
autograd forces / box gradients.  The LAMMPS fixtures that pin the
reference's tests (``tests/data`` of the reference) are converted here too,
keeping the LAMMPS energies/forces beside the reference's outputs.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(REPO, "torch-admp_b200"))
SEED = 1024

from _ref_import import import_reference, reference_root  # noqa: E402

REF_DATA = os.path.join(reference_root(), "tests", "data")

import_reference()
import torch  # noqa: E402

torch.set_default_dtype(torch.float64)
from torch_admp.electrode import (  # noqa: E402
    LAMMPSElectrodeConstraint, PolarizableElectrode, infer, setup_from_lammps)
from torch_admp.nblist import TorchNeighborList  # noqa: E402
from torch_admp.pme import CoulombForceModule  # noqa: E402
from torch_admp.qeq import (  # noqa: E402
    GaussianDampingForceModule, QEqForceModule, SiteForceModule, matinv_optimize, pgrad_optimize)
from torch_admp.utils import calc_grads  # noqa: E402

from admp_b200 import synthetic  # noqa: E402


def T(x, grad=False):
    t = torch.tensor(np.asarray(x), dtype=torch.float64)
    if grad:
        t.requires_grad_(True)
    return t


def save(name, **kw):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in kw.items()})
    print(f"wrote {path} ({os.path.getsize(path) / 1024:.1f} KB)")


def pme_case(name, pos, box, q, rcut, ethresh, kmesh=None, kappa=None, spacing=None,
             rspace=True, kspace=True, slab=False, axis=2, store_pairs=True):
    p = T(pos, True)
    b = T(box, True)
    nb = TorchNeighborList(rcut)
    pairs = nb(p, b)
    ds = nb.get_ds()
    bs = nb.get_buffer_scales()
    m = CoulombForceModule(rcut=rcut, ethresh=ethresh, kmesh=kmesh, kappa=kappa, spacing=spacing,
                           rspace=rspace, kspace=kspace, slab_corr=slab, slab_axis=axis)
    E = m(p, b, pairs, ds, bs, {"charge": T(q)})
    gp, gb = torch.autograd.grad(E.sum(), [p, b])
    # gradient w.r.t. the caller's ds and charges (drop-in contract)
    p2 = T(pos)
    qq = T(q, True)
    ds2 = ds.detach().clone().requires_grad_(True)
    E2 = m(p2, T(box), pairs, ds2, bs, {"charge": qq})
    gds, gq = torch.autograd.grad(E2.sum(), [ds2, qq], allow_unused=True)
    gds = torch.zeros_like(ds2) if gds is None else gds
    extra = {}
    if store_pairs:
        extra = dict(pairs=pairs.numpy(), ds=ds.detach().numpy(), bs=bs.numpy(), dE_dds=gds.numpy())
    save(name, pos=pos, box=box, q=q, rcut=rcut, ethresh=ethresh, kappa=m.kappa,
         kmesh=m._kmesh.numpy(), E=E.detach().numpy(), forces=-gp.numpy(), box_grad=gb.numpy(),
         dE_dq=gq.numpy(), n_pairs=pairs.shape[0], **extra,
         E_real=np.asarray(m.real_energy.detach()).ravel(),
         E_recip=np.asarray(m.reciprocal_energy.detach()).ravel(),
         E_self=np.asarray(m.self_energy.detach()).ravel(),
         E_nn=np.asarray(m.non_neutral_energy.detach()).ravel(),
         E_slab=np.asarray(m.slab_corr_energy.detach()).ravel(),
         rspace=rspace, kspace=kspace, slab=slab, axis=axis,
         kmesh_arg=np.asarray(kmesh if kmesh is not None else -1),
         spacing_arg=np.asarray(spacing if spacing is not None else -1.0))


def case_pme_small():
    rng = np.random.default_rng(SEED)
    n, L = 100, 20.0
    q = rng.uniform(-1.0, 1.0, n)
    q -= q.mean()
    pos = rng.random((n, 3)) * L
    pme_case("pme_small", pos, np.diag([L] * 3), q, 5.0, 5e-6)


def case_pme_cfg1():
    pos, box, q = synthetic.random_charges_system(1536, 25.0, SEED)
    pme_case("pme_cfg1", pos, box, q, 6.0, 5e-4, kmesh=32, store_pairs=False)


def case_pme_triclinic():
    rng = np.random.default_rng(SEED + 1)
    n = 150
    box = np.array([[18.0, 0.0, 0.0], [2.5, 17.0, 0.0], [-1.5, 3.0, 19.0]])
    f = rng.random((n, 3))
    pos = f @ box + rng.normal(0, 0.5, (n, 3))     # some atoms outside the cell
    q = rng.uniform(-1.0, 1.0, n)                  # non-neutral on purpose
    pme_case("pme_triclinic", pos, box, q, 4.0, 1e-5, kmesh=[20, 21, 24])


def case_pme_kspace():
    # reference test_autodiff.py:139-172 style: kappa 0.5, spacing 0.4, no real space
    rng = np.random.default_rng(SEED + 2)
    n, L = 60, 9.0
    pos = rng.random((n, 3)) * L
    q = rng.uniform(-1.0, 1.0, n)
    q -= q.mean()
    pme_case("pme_kspace", pos, np.diag([L, L * 1.1, L * 0.9]), q, 4.0, 1e-5, kappa=0.5, spacing=0.4,
             rspace=False)


def case_pme_slab():
    rng = np.random.default_rng(SEED + 3)
    n = 120
    box = np.diag([14.0, 15.0, 45.0])
    pos = rng.random((n, 3)) * [14.0, 15.0, 15.0]
    q = rng.uniform(-1.0, 1.0, n)
    pme_case("pme_slab", pos, box, q, 5.0, 1e-5, kmesh=[18, 20, 56], slab=True, axis=2)


def read_lammps_data(path):
    """Atoms section of a LAMMPS data file (atom_style full): id mol type q x y z."""
    lines = open(path).read().splitlines()
    lo_hi = {}
    atoms = []
    in_atoms = False
    for ln in lines:
        s = ln.split()
        if len(s) >= 4 and s[2].endswith("lo") and s[3].endswith("hi"):
            lo_hi[s[2][0]] = (float(s[0]), float(s[1]))
        if ln.strip().startswith("Atoms"):
            in_atoms = True
            continue
        if in_atoms:
            if not s:
                if atoms:
                    break
                continue
            if s[0].isalpha():
                break
            atoms.append([float(v) for v in s[:7]])
    a = np.array(sorted(atoms, key=lambda r: r[0]))
    box = np.diag([lo_hi[c][1] - lo_hi[c][0] for c in "xyz"])
    return a[:, 4:7], a[:, 3], box


def read_lammps_dump(path):
    """Last frame of a LAMMPS custom dump: returns dict of columns and the box."""
    lines = open(path).read().splitlines()
    starts = [i for i, l in enumerate(lines) if l.startswith("ITEM: TIMESTEP")]
    fr = lines[starts[-1]:]
    n = int(fr[3])
    bounds = np.array([[float(v) for v in fr[5 + k].split()[:2]] for k in range(3)])
    cols = fr[8].split()[2:]
    rows = [l.split() for l in fr[9:9 + n]]
    out = {}
    for c_i, c in enumerate(cols):
        if c == "element":
            out[c] = np.array([r[c_i] for r in rows])
        else:
            out[c] = np.array([float(r[c_i]) for r in rows])
    order = np.argsort(out["id"])
    out = {k: v[order] for k, v in out.items()}
    box = np.diag(bounds[:, 1] - bounds[:, 0])
    return out, box


def case_obc():
    d = os.path.join(REF_DATA, "lmp_coul_obc")
    pos, q, _ = read_lammps_data(os.path.join(d, "system.data"))
    e_ref = np.loadtxt(os.path.join(d, "thermo.out")).reshape(-1)[1]
    dump, _ = read_lammps_dump(os.path.join(d, "dump.lammpstrj"))
    f_ref = np.stack([dump["fx"], dump["fy"], dump["fz"]], 1)
    p = T(pos, True)
    nb = TorchNeighborList(4.0)
    pairs = nb(p, None)
    m = CoulombForceModule(rcut=5.0, ethresh=1e-5)
    E = m(p, None, pairs, nb.get_ds(), nb.get_buffer_scales(), {"charge": T(q)})
    F = -calc_grads(E, p)
    save("obc", pos=pos, q=q, E_lammps=e_ref, F_lammps=f_ref, E=E.detach().numpy(), forces=F.numpy(),
         pairs=pairs.numpy(), ds=nb.get_ds().detach().numpy(), bs=nb.get_buffer_scales().numpy(), rcut=4.0)


def case_slab_lammps():
    d1 = os.path.join(REF_DATA, "lmp_coul_pbc")
    d2 = os.path.join(REF_DATA, "lmp_coul_pbc_slab_corr")
    pos, q, box = read_lammps_data(os.path.join(d1, "system.data"))
    e1 = np.loadtxt(os.path.join(d1, "thermo.out")).reshape(-1)[1]
    e2 = np.loadtxt(os.path.join(d2, "thermo.out")).reshape(-1)[1]
    f1, _ = read_lammps_dump(os.path.join(d1, "dump.lammpstrj"))
    f2, _ = read_lammps_dump(os.path.join(d2, "dump.lammpstrj"))
    fd = np.stack([f2["fx"] - f1["fx"], f2["fy"] - f1["fy"], f2["fz"] - f1["fz"]], 1)
    p = T(pos, True)
    b = T(box)
    nb = TorchNeighborList(4.0)
    pairs = nb(p, b)
    m = CoulombForceModule(rcut=4.0, ethresh=1e-3, kspace=False, rspace=False, slab_corr=True, slab_axis=2)
    E = m(p, b, pairs, nb.get_ds(), nb.get_buffer_scales(), {"charge": T(q)})
    F = -calc_grads(E, p)
    save("slab_lammps", pos=pos, q=q, box=box, E_lammps=e2 - e1, F_lammps=fd, E=E.detach().numpy(),
         forces=F.numpy())


def case_damping_site():
    rng = np.random.default_rng(SEED + 4)
    n, L = 80, 12.0
    pos = rng.random((n, 3)) * L
    q = rng.uniform(-1, 1, n)
    eta = rng.uniform(0.4, 1.2, n)
    eta[3] = 0.0          # zero-width site exercises safe_inverse / 1e-10 floor
    chi = rng.uniform(3, 9, n)
    hard = rng.uniform(5, 15, n)
    p = T(pos, True)
    b = T(np.diag([L] * 3))
    nb = TorchNeighborList(5.0)
    pairs = nb(p, b)
    ds = nb.get_ds()
    bs = nb.get_buffer_scales()
    tq, te, tc, th = T(q, True), T(eta, True), T(chi, True), T(hard, True)
    Ed = GaussianDampingForceModule()(p, b, pairs, ds, bs, {"charge": tq, "eta": te})
    gp, gq, ge = torch.autograd.grad(Ed.sum(), [p, tq, te])
    Es = SiteForceModule()(p, b, pairs, ds, bs, {"charge": tq, "chi": tc, "hardness": th})
    gsq, gc, gh = torch.autograd.grad(Es.sum(), [tq, tc, th])
    save("damping_site", pos=pos, box=np.diag([L] * 3), q=q, eta=eta, chi=chi, hardness=hard,
         pairs=pairs.numpy(), ds=ds.detach().numpy(), bs=bs.numpy(),
         E_damp=Ed.detach().numpy(), F_damp=-gp.numpy(), dq_damp=gq.numpy(), deta_damp=ge.numpy(),
         E_site=Es.detach().numpy(), dq_site=gsq.numpy(), dchi=gc.numpy(), dhard=gh.numpy())


def qeq_inputs_small():
    # reference test_qeq_numerical.py:163-220 setup
    rng = np.random.default_rng(SEED + 5)
    n, L = 100, 20.0
    pos = rng.random((n, 3)) * L
    chi = rng.random(n)
    return pos, np.diag([L] * 3), chi, np.zeros(n), np.ones(n) * 0.5


def run_qeq(pos, box, chi, hard, eta, rcut, ethresh, kmesh=None, methods=("matinv", "quadratic"),
            eps=1e-6, max_iter=100):
    p = T(pos, True)
    b = T(box)
    nb = TorchNeighborList(rcut)
    pairs = nb(p, b)
    ds = nb.get_ds()
    bs = nb.get_buffer_scales()
    n = pos.shape[0]
    C = torch.ones((1, n))
    cv = torch.zeros(1)
    out = {"pairs": pairs.numpy(), "ds": ds.detach().numpy(), "bs": bs.numpy()}
    for meth in methods:
        mod = QEqForceModule(rcut, ethresh, kmesh=kmesh, eps=eps, ls_eps=eps, max_iter=max_iter)
        t0 = time.time()
        if meth == "matinv":
            E, q = matinv_optimize(mod, p, b, T(chi), T(hard), T(eta), pairs, ds, bs, C, cv)
        else:
            E, q = pgrad_optimize(mod, torch.zeros(n), p, b, T(chi), T(hard), T(eta), pairs, ds, bs, C, cv,
                                  reinit_q=True, method=meth)
            out[f"iters_{meth}"] = mod.converge_iter
        F = -torch.autograd.grad(E.sum(), p, retain_graph=True)[0]
        out[f"q_{meth}"] = q.detach().numpy()
        out[f"E_{meth}"] = E.detach().numpy()
        out[f"F_{meth}"] = F.numpy()
        out[f"time_{meth}"] = time.time() - t0
        print(meth, "E", float(E.sum()), "t", time.time() - t0, flush=True)
    return out


def case_qeq_small():
    pos, box, chi, hard, eta = qeq_inputs_small()
    out = run_qeq(pos, box, chi, hard, eta, 5.0, 1e-6)
    save("qeq_small", pos=pos, box=box, chi=chi, hardness=hard, eta=eta, rcut=5.0, ethresh=1e-6, **out)


def case_qeq_water_small():
    pos, box, chi, hard, eta, _ = synthetic.water_system(64, 12.4, SEED + 6)
    out = run_qeq(pos, box, chi, hard, eta, 6.0, 5e-4, kmesh=20)
    save("qeq_water_small", pos=pos, box=box, chi=chi, hardness=hard, eta=eta, rcut=6.0, ethresh=5e-4,
         kmesh=20, **out)


def case_qeq_water_cfg2():
    pos, box, chi, hard, eta, _ = synthetic.water_system(1000, 31.0, SEED)
    out = run_qeq(pos, box, chi, hard, eta, 6.0, 5e-4, kmesh=48, methods=("quadratic",), eps=1e-7,
                  max_iter=200)
    save("qeq_water_cfg2", pos=pos, box=box, chi=chi, hardness=hard, eta=eta, rcut=6.0, ethresh=5e-4,
         kmesh=48, **out)


ELECTRODE_CASES = {
    # name: (slab_corr, ffield, [(first, last, value, mode)], symm)
    "lmp_conp_slab_2d": (True, False, [(0, 108, 20.0, "conp"), (108, 216, 0.0, "conp")], True),
    "lmp_conp_slab_3d": (False, True, [(0, 108, 20.0, "conp"), (108, 216, 0.0, "conp")], True),
    "lmp_conp_interface_2d_bias": (True, False, [(0, 108, 20.0, "conp"), (108, 216, 0.0, "conp")], True),
    "lmp_conq_interface_2d_pzc": (True, False, [(0, 216, 0.0, "conq")], False),
    # the remaining LAMMPS fixtures of test_electrode_conp.py / test_electrode_conq.py, with their settings
    "lmp_conp_interface_2d_pzc": (True, False, [(0, 108, 0.0, "conp"), (108, 216, 0.0, "conp")], True),
    "lmp_conp_interface_3d_pzc": (False, True, [(0, 108, 0.0, "conp"), (108, 216, 0.0, "conp")], True),
    "lmp_conp_interface_3d_bias": (False, True, [(0, 108, 20.0, "conp"), (108, 216, 0.0, "conp")], True),
    "lmp_conq_interface_3d_pzc": (False, False, [(0, 216, 0.0, "conq")], False),
    "lmp_conq_interface_2d_edl": (True, False, [(0, 216, -10.0, "conq")], False),
    "lmp_conq_interface_3d_edl": (False, False, [(0, 216, -10.0, "conq")], False),
    "lmp_conq_interface_2d_bias": (True, False, [(0, 108, -10.0, "conq"), (108, 216, 10.0, "conq")], False),
}


def case_electrode(name):
    slab, ffield, cons, symm = ELECTRODE_CASES[name]
    dump, box = read_lammps_dump(os.path.join(REF_DATA, name, "dump.lammpstrj"))
    pos = np.stack([dump["xu"], dump["yu"], dump["zu"]], 1)
    q = dump["q"]
    f_ref = np.stack([dump["fx"], dump["fy"], dump["fz"]], 1)
    cell = box.copy()
    if slab:
        cell[2, 2] *= 3.0
    rcut = 5.0
    calc = PolarizableElectrode(rcut=rcut, kappa=0.5, slab_corr=slab, eps=1e-6, ls_eps=1e-6, max_iter=100,
                                ethresh=1e-6)
    p = T(pos, True)
    b = T(cell)
    ch = T(q, True)
    nb = TorchNeighborList(rcut)
    pairs = nb(p, b)
    ds = nb.get_ds()
    bs = nb.get_buffer_scales()
    lc = [LAMMPSElectrodeConstraint(indices=np.arange(a, z), value=v, mode=md, eta=1.6, ffield=ffield)
          for (a, z, v, md) in cons]
    data = setup_from_lammps(len(q), lc, symm)
    t0 = time.time()
    E, F, qo = infer(calc, p, b, ch, pairs, ds, bs, *data, method="matinv")
    print(name, "matinv", time.time() - t0, "max|dF| vs lammps", np.abs(F.detach().numpy() - f_ref).max(),
          flush=True)
    save("electrode_" + name.replace("lmp_", ""), pos=pos, box=cell, q_lammps=q, F_lammps=f_ref,
         E=np.asarray(E.detach()), forces=F.detach().numpy(), q_ref=qo.detach().numpy(),
         kmesh=calc.submodels["coulomb"]._kmesh.numpy(), slab_corr=slab, ffield=ffield, symm=symm,
         cons=np.array([[a, z, v, 0 if md == "conp" else 1] for (a, z, v, md) in cons]),
         lammps_eta=1.6, rcut=rcut, kappa=0.5, ethresh=1e-6)


def electrode_cfg3_inputs(n_side=24, n_ions=3000, seed=SEED):
    """Two fcc(111) slabs of 2 x n_side^2 atoms, n_ions +-1 ions in a 40 A gap,
    Lz = 3 x slab extent, electrode Gaussian width 0.5 A (LAMMPS eta sqrt 2),
    CONP at 1 V (top) and 0 V (bottom), total electrode charge 0 (symm)."""
    pos, box, q, top, bot = synthetic.electrode_system(seed, n_side=n_side, n_ions=n_ions)
    cons = [(int(top[0]), int(top[-1]) + 1, 1.0, "conp"), (int(bot[0]), int(bot[-1]) + 1, 0.0, "conp")]
    return pos, box, q, cons


def case_electrode_cfg3():
    """Constant-potential electrodes at their stated size: 2 x 1,152 electrode
    atoms, 3,000 ions, 64 x 64 x 160 mesh, slab correction along z."""
    pos, box, q, cons = electrode_cfg3_inputs()
    rcut, ethresh, kmesh = 6.0, 5e-4, [64, 64, 160]
    calc = PolarizableElectrode(rcut=rcut, ethresh=ethresh, kmesh=kmesh, slab_corr=True, eps=1e-8, ls_eps=1e-8,
                                max_iter=400)
    p = T(pos, True)
    b = T(box)
    ch = T(q, True)
    nb = TorchNeighborList(rcut)
    pairs = nb(p, b)
    lc = [LAMMPSElectrodeConstraint(indices=np.arange(a, z), value=v, mode=md, eta=np.sqrt(2.0)) for (a, z, v, md)
          in cons]
    data = setup_from_lammps(len(q), lc, True)
    t0 = time.time()
    E, F, qo = infer(calc, p, b, ch, pairs, nb.get_ds(), nb.get_buffer_scales(), *data, method="lbfgs")
    print("electrode_cfg3 lbfgs", time.time() - t0, "s, E", float(E), flush=True)
    save("electrode_cfg3", pos=pos, box=box, q_in=q, E=np.asarray(E.detach()), forces=F.detach().numpy(),
         q_ref=qo.detach().numpy(), cons=np.array([[a, z, v, 0] for (a, z, v, md) in cons]), lammps_eta=np.sqrt(2.0),
         rcut=rcut, ethresh=ethresh, kmesh=np.array(kmesh), eps=1e-8, time_ref_s=time.time() - t0,
         threads=torch.get_num_threads())


def case_qeq_cfg4():
    """Energy gradients of the differentiation batch at the solved charges:
    frames 0 and 1 of the jittered 1,000-water system (3,000 atoms, 31 A box,
    48^3 mesh, rc 6).  The reference evaluates E at the detached optimum
    (qeq.py:1262-1268), so its autograd gradient is the total derivative
    (the charge response drops out at the constrained minimum).  eps 1e-8:
    at 1e-9 the reference's nonlinear CG ran 374 iterations on frame 0 and
    left the total-charge constraint (E -2760 instead of -209.9 eV)."""
    pos_f, box_f, chi, hard, eta, _ = synthetic.water_frames(2, SEED)
    out = {}
    for f in range(2):
        p = T(pos_f[f], True)
        b = T(box_f[f], True)
        c, h, e = T(chi, True), T(hard, True), T(eta, True)
        nb = TorchNeighborList(6.0)
        pairs = nb(p, b)
        ds = nb.get_ds()
        bs = nb.get_buffer_scales()
        n = pos_f.shape[1]
        mod = QEqForceModule(6.0, 5e-4, kmesh=48, eps=1e-8, ls_eps=1e-8, max_iter=400)
        t0 = time.time()
        E, q = pgrad_optimize(mod, torch.zeros(n), p, b, c, h, e, pairs, ds, bs, torch.ones((1, n)), torch.zeros(1),
                              reinit_q=True, method="quadratic")
        g = torch.autograd.grad(E.sum(), [p, b, c, h, e])
        assert 0 <= mod.converge_iter < 400 and abs(float(q.sum())) < 1e-9
        print("qeq_cfg4 frame", f, "iters", mod.converge_iter, "t", time.time() - t0, "E", float(E.sum()), flush=True)
        for k, v in zip(("dpos", "dbox", "dchi", "dhard", "deta"), g):
            out[f"{k}_{f}"] = v.numpy()
        out[f"E_{f}"] = E.detach().numpy()
        out[f"q_{f}"] = q.detach().numpy()
        out[f"iters_{f}"] = mod.converge_iter
    save("qeq_cfg4", pos=pos_f, box=box_f, chi=chi, hardness=hard, eta=eta, rcut=6.0, ethresh=5e-4, kmesh=48, **out)


def case_qeq_dq_dchi():
    """dq/dchi through the reference's dense KKT solve, which stays
    differentiable in chi (QEqForceModule.solve_matrix_inversion,
    qeq.py:517-607): 64 waters (192 atoms) in a 12.4 A box, loss
    L = sum_i w_i q_i with seeded weights w."""
    pos, box, chi, hard, eta, _ = synthetic.water_system(64, 12.4, SEED + 6)
    n = pos.shape[0]
    w = np.random.default_rng(SEED + 8).normal(size=n)
    p, b = T(pos), T(box)
    c = T(chi, True)
    nb = TorchNeighborList(6.0)
    pairs = nb(p, b)
    mod = QEqForceModule(6.0, 5e-4, kmesh=20)
    E, q, _, _ = mod.solve_matrix_inversion(p, b, c, T(hard), T(eta), pairs, nb.get_ds(), nb.get_buffer_scales(),
                                           torch.ones((1, n)), torch.zeros(1))
    loss = (q * T(w)).sum()
    (gchi,) = torch.autograd.grad(loss, [c])
    save("qeq_dq_dchi", pos=pos, box=box, chi=chi, hardness=hard, eta=eta, w=w, q=q.detach().numpy(),
         dL_dchi=gchi.numpy(), rcut=6.0, ethresh=5e-4, kmesh=20)


def case_ewald_params():
    """setup_ewald_parameters (pme.py:564-658) over both methods, several
    cut-offs, thresholds, spacings and orthogonal boxes."""
    from torch_admp.pme import setup_ewald_parameters
    rows = []
    for rcut in (4.0, 5.0, 6.0, 9.5):
        for thr in (1e-3, 5e-4, 1e-5, 1e-7):
            for L in ((10.0, 10.0, 10.0), (25.0, 31.0, 58.5), (69.24, 59.96, 140.1)):
                box = np.diag(L)
                k, kx, ky, kz = setup_ewald_parameters(rcut, box, thr, method="openmm")
                rows.append([0, rcut, thr, 0.0, *L, k, kx, ky, kz])
                for sp in (0.5, 1.0, 1.37):
                    k, kx, ky, kz = setup_ewald_parameters(rcut, box, thr, spacing=sp, method="gromacs")
                    rows.append([1, rcut, thr, sp, *L, k, kx, ky, kz])
    save("ewald_params", rows=np.array(rows, dtype=np.float64),
         columns=np.array(["method", "rcut", "threshold", "spacing", "Lx", "Ly", "Lz", "kappa", "kx", "ky", "kz"]))


def case_nblist():
    rng = np.random.default_rng(SEED + 7)
    out = {}
    for tag, box in [("cubic", np.diag([13.0, 13.0, 13.0])),
                     ("tric", np.array([[14.0, 0.0, 0.0], [3.0, 13.5, 0.0], [1.0, -2.0, 15.0]]))]:
        n = 250
        pos = rng.random((n, 3)) @ box + rng.normal(0, 2.0, (n, 3))
        p = T(pos, True)
        b = T(box, True)
        nb = TorchNeighborList(6.0)
        pairs = nb(p, b)
        ds = nb.get_ds()
        gp, gb = torch.autograd.grad((ds * torch.linspace(0.5, 1.5, ds.shape[0])).sum(), [p, b])
        out[f"{tag}_pos"] = pos
        out[f"{tag}_box"] = box
        out[f"{tag}_pairs"] = pairs.numpy()
        out[f"{tag}_ds"] = ds.detach().numpy()
        out[f"{tag}_bs"] = nb.get_buffer_scales().numpy()
        out[f"{tag}_gpos"] = gp.numpy()
        out[f"{tag}_gbox"] = gb.numpy()
    save("nblist", **out)


CASES = {
    "pme_small": case_pme_small, "pme_cfg1": case_pme_cfg1, "pme_triclinic": case_pme_triclinic,
    "pme_kspace": case_pme_kspace, "pme_slab": case_pme_slab, "obc": case_obc,
    "slab_lammps": case_slab_lammps, "damping_site": case_damping_site, "qeq_small": case_qeq_small,
    "qeq_water_small": case_qeq_water_small, "qeq_water_cfg2": case_qeq_water_cfg2, "nblist": case_nblist,
    "electrode_cfg3": case_electrode_cfg3, "ewald_params": case_ewald_params,
    "qeq_cfg4": case_qeq_cfg4, "qeq_dq_dchi": case_qeq_dq_dchi,
}
for _n in ELECTRODE_CASES:
    CASES["electrode_" + _n] = (lambda nm: (lambda: case_electrode(nm)))(_n)

if __name__ == "__main__":
    torch.set_num_threads(os.cpu_count())
    names = sys.argv[1:] or list(CASES)
    for nm in names:
        t0 = time.time()
        CASES[nm]()
        print(f"[{nm}] {time.time() - t0:.1f}s", flush=True)
