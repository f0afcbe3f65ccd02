"""The drop-in modules compile with torch.jit.script and survive save / load,
as the reference's do (test_jit.py of torch-admp): their forward passes call
the TorchScript operators torch.ops.admp_b200.* (a C++ extension over the C
ABI).  Compiling needs no GPU; running them does (test_gpu_jit.py)."""
import io

import pytest
import torch


def _modules():
    from admp_b200.pme import CoulombForceModule
    from admp_b200.qeq import GaussianDampingForceModule, QEqForceModule, SiteForceModule
    return {
        "coulomb": CoulombForceModule(rcut=4.0, ethresh=1e-5),
        "coulomb_slab_x": CoulombForceModule(rcut=4.0, ethresh=1e-5, slab_corr=True, slab_axis=0),
        "coulomb_kmesh": CoulombForceModule(rcut=4.0, ethresh=1e-5, kmesh=[10, 12, 14]),
        "coulomb_spacing": CoulombForceModule(rcut=4.0, spacing=0.5),
        "damping": GaussianDampingForceModule(),
        "site": SiteForceModule(),
        "qeq": QEqForceModule(rcut=4.0, ethresh=1e-5),
        "qeq_nodamp_slab": QEqForceModule(rcut=4.0, ethresh=1e-5, damping=False, slab_corr=True),
    }


@pytest.mark.parametrize("name", list(_modules()))
def test_modules_script_save_load(name):
    m = _modules()[name]
    sm = torch.jit.script(m)
    buf = io.BytesIO()
    torch.jit.save(sm, buf)
    buf.seek(0)
    loaded = torch.jit.load(buf)
    assert hasattr(loaded, "forward")
    if name.startswith("qeq"):
        assert hasattr(loaded, "func_energy") and hasattr(loaded, "optimality")


def test_scripted_module_rejects_cpu_tensors():
    from admp_b200.pme import CoulombForceModule
    sm = torch.jit.script(CoulombForceModule(rcut=4.0, ethresh=1e-5))
    pos = torch.rand(10, 3, dtype=torch.float64) * 10
    box = torch.eye(3, dtype=torch.float64) * 10
    pairs = torch.tensor([[0, 1], [1, 0]])
    ds = torch.ones(2, dtype=torch.float64)
    bs = torch.tensor([1.0, 0.0], dtype=torch.float64)
    with pytest.raises(Exception, match="CUDA"):
        sm(pos, box, pairs, ds, bs, {"charge": torch.zeros(10, dtype=torch.float64)})
