"""The "cuda" 6-face diffusion plugin (cdb_diff6_*) against the oracle's
numpy restatement of CUDADiffusion (oracle/diff6.py): face conductivities
and dVm on a box with rotated fibres and on an irregular mask, within 1e-12
of the largest |dVm| (the GPU may contract products into FMAs).

The face-conductivity table is pinned to the reference's own code: the
oracle build constructs the reference's CUDADiffusion (its constructor
builds the table on the host, elec/CUDADiffusion.cc:73-122), and both the
restatement (CPU) and the plugin (GPU) reproduce it bit for bit.  The
reference's kernel (diff_6face_v1) returns from threads before a
__syncthreads unless the local grid's y and z sizes are 30 k + 2; on such
tissues the reference's own "cuda" Diffusion runs on the GPU
(oracle/_ref/ref_gpu_diff6) and the plugin's dVm is checked against it."""
import numpy as np
import pytest

from cardioid_b200 import tissue


def _tissues():
    box = tissue.box(11, 9, 7, seed=3)
    x, y, z = box.tuples()
    keep = ~((x >= 4) & (x <= 6) & (y >= 3) & (y <= 5) & (z >= 2) & (z <= 4))
    keep &= ~((x == 10) & (y == 0))
    masked = tissue.Tissue(box.nx, box.ny, box.nz, box.dx, box.dy, box.dz, box.gid[keep], box.cell_type[keep],
                           box.sigma[keep], box.vm0[keep], [])
    return {"box": box, "masked": masked}


def _ref_built():
    from oracle import refsim
    return refsim.available()


def _reference_faces(t):
    """The reference CUDADiffusion's face table at t's cells (diffusion
    scale t.diffusion_scale)."""
    from golden.make_golden import reference_sim
    sim = reference_sim(t)
    try:
        return sim.diff6_face_sigma(t.tuples())
    finally:
        sim.close()


@pytest.mark.skipif(not _ref_built(), reason="needs the reference build (oracle/_ref)")
@pytest.mark.parametrize("kind", ["box", "masked"])
def test_oracle_face_table_is_the_references(kind):
    from oracle import diff6
    t = _tissues()[kind]
    ref = _reference_faces(t)
    np.testing.assert_array_equal(diff6.face_sigma(t, t.diffusion_scale), ref)


def test_oracle_face_rule_on_a_uniform_box():
    from oracle import diff6
    t = tissue.box(5, 4, 3, seed=1)
    t.sigma = np.tile([2.0, 0.5, 0.0, 3.0, 0.0, 4.0], (t.n, 1))
    f = diff6.face_sigma(t, 1.0)
    x, y, z = t.tuples()
    inner = (x > 0) & (y > 0) & (y < 3) & (z > 0) & (z < 2)
    h = t.dx
    np.testing.assert_allclose(f[inner, 0, 0], 2.0 * h * h / h / h ** 3)
    np.testing.assert_allclose(f[inner, 0, 1], 0.5 * h * h / h / h ** 3)
    assert (f[x == 0, 0, :] == 0).all()          # no left neighbour
    # a constant field has no flux
    np.testing.assert_allclose(diff6.calc(t, np.full(t.n, -80.0), 1.0), 0.0, atol=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["box", "masked"])
def test_diff6_plugin_matches_oracle(cdb_lib, kind):
    import torch
    from cardioid_b200 import plugins
    from oracle import diff6
    t = _tissues()[kind]
    rng = np.random.default_rng(7)
    vm = -80.0 + 40.0 * rng.random(t.n)
    d = plugins.CUDADiffusion(t, 714.2857)
    np.testing.assert_allclose(d.face_sigma(), diff6.face_sigma(t, 714.2857), rtol=1e-15, atol=0)
    if _ref_built():
        d2 = plugins.CUDADiffusion(t, t.diffusion_scale)
        np.testing.assert_array_equal(d2.face_sigma(), _reference_faces(t))
    V = torch.tensor(vm, device="cuda")
    out = torch.empty_like(V)
    d.updateLocalVoltage(V)
    d.calc(out)
    torch.cuda.synchronize()
    ref = diff6.calc(t, vm, 714.2857)
    got = out.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def _tissues30():
    """Tissues whose y and z extents are 30 (local grid 30 k + 2), the only
    shapes the reference kernel runs on without returning from threads
    before its barriers: a rotated-fibre box and the same box with a hole
    and a notch (extents kept)."""
    box = tissue.box(23, 30, 30, seed=4)
    x, y, z = box.tuples()
    keep = ~((x >= 8) & (x <= 14) & (y >= 10) & (y <= 17) & (z >= 5) & (z <= 20))
    keep &= ~((x == 22) & (y < 6))
    masked = tissue.Tissue(box.nx, box.ny, box.nz, box.dx, box.dy, box.dz, box.gid[keep], box.cell_type[keep],
                           box.sigma[keep], box.vm0[keep], [])
    return {"box": box, "masked": masked}


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["box", "masked"])
def test_diff6_plugin_matches_reference_kernel(cdb_lib, oracle_port, kind):
    """The plugin against the reference's own "cuda" Diffusion run on the
    GPU (CUDADiffusion.cc and diff_6face_v1 built from the reference
    sources, oracle/_ref/ref_gpu_diff6): dVm within 1e-12 of the largest
    |dVm| (the two sum the face fluxes in different orders), and the numpy
    restatement within the same bound."""
    import torch
    from cardioid_b200 import plugins
    from oracle import diff6, refgpu
    if not refgpu.diff6_available():
        pytest.skip("oracle/_ref/ref_gpu_diff6 not built (needs the reference checkout at build time)")
    t = _tissues30()[kind]
    rng = np.random.default_rng(11)
    vm = -80.0 + 40.0 * rng.random(t.n)
    ref = refgpu.diff6(t, vm, t.diffusion_scale)
    scale = np.abs(ref).max()
    assert scale > 0
    d = plugins.CUDADiffusion(t, t.diffusion_scale)
    V = torch.tensor(vm, device="cuda")
    out = torch.empty_like(V)
    d.updateLocalVoltage(V)
    d.calc(out)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-12 * scale, np.abs(got - ref).max() / scale
    assert np.abs(diff6.calc(t, vm, t.diffusion_scale) - ref).max() <= 1e-12 * scale
