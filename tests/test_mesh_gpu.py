"""Surface mesher through the C ABI (Mesher, Rendering/Renderer3D/Mesher.cu).

* SDF: the library's computeSDF rounds every operation as the oracle does,
  in the reference's summation order: bit for bit equal to the oracle.
* Marching cubes: the library samples the SDF through the texture unit with
  the reference's sampler settings, the oracle through a model of it; the
  records are matched cube by cube (see mesh_check.py).
* Against the reference's own mesher (recorded fixtures, and live where
  oracle/_ref/libaqmesh.so is present): same cubes, vertices to float
  rounding.
"""
import numpy as np
import pytest

import aquarius_b200 as aq
from mesh_check import compare_meshes, match_records, record_aggregates, used_slots
from oracle_binding import Oracle, RefMesher, mesh_ref_available
from scenes import SCENES, rel_l2

pytestmark = pytest.mark.gpu

GOLDEN_MESH = [("cfg1_16", "ref_cfg1_16"), ("aniso", "ref_aniso")]


def _fluid_at(cfg, positions):
    """A library fluid holding the given (cell-sorted) particle positions."""
    f = aq.Fluid(cfg)
    f.upload_state({"position": np.ascontiguousarray(positions, np.float32)})
    f.run_stage("sort")  # rebuilds the cell tables; a sorted array keeps its order
    return f


def _oracle_state(scene, steps):
    cfg = SCENES[scene]()
    o = Oracle(cfg)
    o.step(steps)
    return cfg, o


def test_mesh_info_matches_oracle():
    for scene in ("cfg1_16", "aniso", "cfg2_32"):
        cfg = SCENES[scene]()
        info = aq.Fluid(cfg).mesh_info()
        d = Oracle(cfg).mesh_dims()
        assert info["sdf"] == d["sdf"] and info["mesh"] == d["mesh"] == (128, 128, 128)
        assert info["h_sdf"] == np.float32(d["h_sdf"]) and info["h_mesh"] == np.float32(d["h_mesh"])


@pytest.mark.parametrize("scene,steps", [("cfg1_16", 4), ("aniso", 3), ("multi_16", 3), ("cfg2_32", 2)])
def test_sdf_is_bit_exact_and_mesh_matches_oracle(scene, steps):
    cfg, o = _oracle_state(scene, steps)
    st = o.get_state(["position"])
    f = _fluid_at(cfg, st["position"])
    np.testing.assert_array_equal(f.download_state(["position"])["position"], st["position"])
    rec = f.download_mesh()
    r = o.mesh()
    np.testing.assert_array_equal(f.download_sdf(), r["sdf"])
    c = compare_meshes(rec, r["records"], r["dims"]["h_mesh"])
    assert abs(c["a"] - c["b"]) <= 5e-4 * c["b"], c
    assert c["matched"] >= 0.995 * c["b"], c
    pairs, _, _ = match_records(rec, r["records"], 0.25 * r["dims"]["h_mesh"])
    ra, rb = rec[pairs[:, 0]], r["records"][pairs[:, 1]]
    u = used_slots(ra)
    dp = np.abs(ra[..., :3] - rb[..., :3]).max(-1)[u] / r["dims"]["h_mesh"]
    assert np.percentile(dp, 50) <= 1e-4 and np.percentile(dp, 99) <= 0.02, np.percentile(dp, [50, 99, 100])


@pytest.mark.parametrize("scene,fixture", GOLDEN_MESH)
def test_mesh_against_reference_fixtures(scene, fixture):
    mz = np.load("tests/golden/ref_mesh.npz")
    pos = np.load(f"tests/golden/{fixture}.npz")[str(mz[f"{scene}/input"])]
    f = _fluid_at(SCENES[scene](), pos)
    rec = f.download_mesh()
    ref_sdf = mz[f"{scene}/sdf"].transpose(2, 1, 0)
    sdf = f.download_sdf()
    assert rel_l2(sdf, ref_sdf) <= 1e-5
    cubes = int(mz[f"{scene}/cubes"])
    assert abs(len(rec) - cubes) <= 2e-4 * cubes
    agg = record_aggregates(rec)
    assert abs(agg["vertices"] - int(mz[f"{scene}/agg/vertices"])) <= 2e-4 * agg["vertices"]
    h_mesh = float(mz[f"{scene}/cell"][1])
    sample = mz[f"{scene}/sample"]
    pairs, _, _ = match_records(sample, rec, 0.25 * h_mesh)
    assert len(pairs) >= 0.995 * len(sample)
    ra, rb = sample[pairs[:, 0]], rec[pairs[:, 1]]
    u = used_slots(ra)
    dp = np.abs(ra[..., :3] - rb[..., :3]).max(-1)[u] / h_mesh
    assert np.percentile(dp, 99) <= 1e-3, np.percentile(dp, [50, 99, 100])


def test_mesh_is_deterministic_and_apis_agree():
    cfg, o = _oracle_state("cfg1_16", 3)
    f = _fluid_at(cfg, o.get_state(["position"])["position"])
    a = f.download_mesh()
    b = f.download_mesh()
    np.testing.assert_array_equal(a, b)
    torch = pytest.importorskip("torch")
    cap = len(a) + 100
    buf = torch.full((cap * 90,), 7.0, dtype=torch.float32, device="cuda")
    n = f.mesh_into(buf.data_ptr(), cap)
    torch.cuda.synchronize()
    host = buf.cpu().numpy().reshape(cap, 15, 6)
    assert n == len(a)
    np.testing.assert_array_equal(host[:n], a)
    assert not host[n:].any()  # cleared past the last record
    # a smaller capacity drops the records past it and still reports the count
    small = torch.zeros((10 * 90,), dtype=torch.float32, device="cuda")
    assert f.mesh_into(small.data_ptr(), 10) == n
    np.testing.assert_array_equal(small.cpu().numpy().reshape(10, 15, 6), a[:10])


def test_mesh_buffer_tail_is_cleared_when_the_mesh_shrinks():
    torch = pytest.importorskip("torch")
    cfg, o = _oracle_state("cfg1_16", 2)
    pos = o.get_state(["position"])["position"]
    f = _fluid_at(cfg, pos)
    cap = 200000
    buf = torch.zeros((cap * 90,), dtype=torch.float32, device="cuda")
    n1 = f.mesh_into(buf.data_ptr(), cap)
    # squeeze every particle into a small ball near the centre: fewer cubes
    c = pos.mean(axis=1, keepdims=True)
    small = (c + 0.2 * (pos - c)).astype(np.float32)
    f.upload_state({"position": small})
    f.run_stage("sort")
    n2 = f.mesh_into(buf.data_ptr(), cap)
    assert 0 < n2 < n1
    host = buf.cpu().numpy().reshape(cap, 15, 6)
    np.testing.assert_array_equal(host[:n2], f.download_mesh())
    assert not host[n2:].any()


def test_unsorted_particles_are_rejected():
    cfg, o = _oracle_state("cfg1_16", 1)
    pos = o.get_state(["position"])["position"]
    f = aq.Fluid(cfg)
    perm = np.random.default_rng(3).permutation(pos.shape[1])
    f.upload_state({"position": np.ascontiguousarray(pos[:, perm])})
    with pytest.raises(aq.AquariusError):
        f.download_mesh()
    f.run_stage("sort")
    assert len(f.download_mesh()) > 0


def test_mesh_leaves_the_step_unchanged():
    """Meshing between steps does not reorder or touch the fluid's state."""
    cfg = SCENES["cfg1_16"]()
    a, b = aq.Fluid(cfg), aq.Fluid(cfg)
    for _ in range(3):
        a.step(1)
        b.step(1)
        a.download_mesh()
    sa, sb = a.download_state(), b.download_state()
    for k in sa:
        np.testing.assert_array_equal(sa[k], sb[k], err_msg=k)


@pytest.mark.skipif(not mesh_ref_available(), reason="reference mesher build (oracle/_ref) not present")
@pytest.mark.parametrize("scene,steps", [("cfg1_16", 3), ("cfg2_32", 2)])
def test_mesh_against_live_reference(scene, steps):
    cfg = SCENES[scene]()
    f = aq.Fluid(cfg)
    f.step(steps)
    pos = f.download_state(["position"])["position"]
    rec = f.download_mesh()
    h = float(np.float32(cfg.domain_size) / np.float32(cfg.size_y))
    m = RefMesher((cfg.size_x, cfg.size_y, cfg.size_z), h, pos.shape[1])
    r = m.mesh(pos, capacity_cubes=len(rec) + 4096)
    m.close()
    assert rel_l2(f.download_sdf(), r["sdf"].transpose(2, 1, 0)) <= 1e-5
    c = compare_meshes(rec, r["records"], m.h_mesh)
    assert abs(c["a"] - c["b"]) <= 2e-4 * c["b"], c
    assert c["matched"] >= 0.998 * c["b"], c
    pairs, _, _ = match_records(rec, r["records"], 0.25 * m.h_mesh)
    ra, rb = rec[pairs[:, 0]], r["records"][pairs[:, 1]]
    u = used_slots(ra)
    dp = np.abs(ra[..., :3] - rb[..., :3]).max(-1)[u] / m.h_mesh
    assert np.percentile(dp, 99) <= 1e-3, np.percentile(dp, [50, 99, 100])


@pytest.mark.skipif(not mesh_ref_available(), reason="reference mesher build (oracle/_ref) not present")
def test_mesh_time_vs_reference_mesher(capsys):
    """The 128^3 ball drop after 3 steps (5.2M particles, SDF 259^3, mesh
    128^3) on the same GPU: ours into a device buffer (CUDA events around the
    calls, each ending with a host read of the count) against the reference's
    Mesher::mesh (CUDA events around the call, its own syncs included)."""
    import bench
    torch = pytest.importorskip("torch")

    f = aq.Fluid(bench.workload_config(128, "zero"))
    f.step(3)
    f.synchronize()
    pos = f.download_state(["position"])["position"]
    cap = 1 << 19
    buf = torch.empty((cap * 90,), dtype=torch.float32, device="cuda")
    for _ in range(2):
        cubes = f.mesh_into(buf.data_ptr(), cap)
    reps = 5
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        f.mesh_into(buf.data_ptr(), cap)
    e1.record()
    e1.synchronize()
    ours = e0.elapsed_time(e1) / reps
    del buf
    h = float(np.float32(10.0) / np.float32(128))
    m = RefMesher((128, 128, 128), h, pos.shape[1])
    ref = []
    for i in range(reps + 1):
        r = m.mesh(pos, capacity_cubes=1, want_sdf=False)
        if i:
            ref.append(r["ms"])
    m.close()
    ref = float(np.mean(ref))
    with capsys.disabled():
        print(f"\nmesh 128^3 workload: ours {ours:.3f} ms/mesh, reference Mesher::mesh {ref:.3f} ms, "
              f"cubes {cubes} vs {r['cubes']}")
    assert abs(cubes - r["cubes"]) <= 2e-4 * r["cubes"]
    assert ours < ref
