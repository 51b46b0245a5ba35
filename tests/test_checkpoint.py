"""Checkpoint / restart (the reference's restart example) : file format on the host, and a
resumed density-matrix run on the GPU equal to an uninterrupted one."""
import os

import numpy as np
import pytest

from oracle import mps_ref as R


@pytest.mark.parametrize("ext", [".npz", ".mat"])
def test_checkpoint_round_trip_host(tmp_path, ext):
    """Both containers: NumPy .npz, and a MAT v5 file with the reference writer's variable
    names and the MPS as a cell array of complex sites (readable by MATLAB / MAT.jl / scipy)."""
    from mpsb200 import checkpoint as CK
    rng = np.random.default_rng(1)
    sites, dims = R.mpsrandom(6, 8, 4, rng)
    f = str(tmp_path / ("run_temp" + ext))
    CK.write_data_file(f, {"rho": sites, "i_last": 17, "dt": 0.005, "tr_rho": np.array([1.0 + 0j, 0.99]),
                           "rj": np.arange(6.0)})
    st = CK.read_data_file(f, device=False)
    assert st["i_last"] == 17 and st["dt"] == 0.005
    assert np.array_equal(st["tr_rho"], [1.0 + 0j, 0.99]) and np.array_equal(st["rj"], np.arange(6.0))
    assert len(st["rho"]) == 6 and all(np.array_equal(a, b) for a, b in zip(st["rho"], sites))
    assert not os.path.exists(f + ".tmp")
    with pytest.raises(ValueError):
        CK.write_data_file(f, {"a/b": 1})
    if ext == ".mat":   # what a MAT reader sees: a column cell array of 3-d complex sites
        import scipy.io
        raw = scipy.io.loadmat(f)
        assert raw["rho"].shape == (6, 1) and raw["rho"][2, 0].shape == sites[2].shape
        assert raw["i_last"].shape == (1, 1)


@pytest.mark.parametrize("ext", [".npz", ".mat"])
def test_checkpoint_keeps_field_shapes(tmp_path, ext):
    """Size-1 arrays and 1 x n matrices read back with their own shapes (a run checkpointed
    before its second measurement holds exactly such observation arrays)."""
    from mpsb200 import checkpoint as CK
    f = str(tmp_path / ("obs" + ext))
    fields = {"tr_rho": np.array([1.0 + 0j]), "see": np.array([[0.0, 1.0, 2.0, 3.0]]), "spm": np.zeros((1, 1), complex),
              "col": np.arange(3.0).reshape(3, 1), "cube": np.arange(24.0).reshape(2, 3, 4), "n": 5, "x": 0.25}
    CK.write_data_file(f, fields)
    st = CK.read_data_file(f, device=False)
    for k, v in fields.items():
        assert np.shape(st[k]) == np.shape(v), k
        assert np.array_equal(np.asarray(st[k]), np.asarray(v)), k
    assert isinstance(st["n"], int) and isinstance(st["x"], float)


@pytest.mark.gpu
@pytest.mark.parametrize("ext", [".npz", ".mat"])
def test_resume_from_a_single_observation_row(gpu_ctx, tmp_path, ext):
    """checkpoint_int < measure_int: the first checkpoint holds one observation row."""
    from mpsb200 import drivers as GDR, models as GM
    na, chi, dt = 6, 16, 0.005
    pg = GM.WaveguideChain(na, gam_eg=0.1, omega=0.5, gam_phi=0.1)
    b_ref, obs_ref = GDR.run_density(pg, chi, dt, 4, w=8, measure_int=2, ctx=gpu_ctx)
    f = str(tmp_path / ("rho1_temp" + ext))
    GDR.run_density(pg, chi, dt, 1, w=8, measure_int=2, ctx=gpu_ctx, checkpoint=f, checkpoint_int=1)
    b, obs = GDR.run_density(pg, chi, dt, 4, w=8, measure_int=2, ctx=gpu_ctx, checkpoint=f)
    assert all(np.array_equal(a, c) for a, c in zip(b.rho.sites(), b_ref.rho.sites()))
    assert len(obs) == len(obs_ref)


@pytest.mark.gpu
@pytest.mark.parametrize("ext", [".npz", ".mat"])
def test_resumed_density_run_equals_uninterrupted(gpu_ctx, tmp_path, ext):
    from mpsb200 import drivers as GDR, models as GM
    na, chi, dt, n = 6, 16, 0.005, 8
    pg = GM.WaveguideChain(na, gam_eg=0.1, omega=0.5, gam_phi=0.1)
    b_ref, obs_ref = GDR.run_density(pg, chi, dt, n, w=8, measure_int=2, ctx=gpu_ctx)
    f = str(tmp_path / ("rho_temp" + ext))
    GDR.run_density(pg, chi, dt, 4, w=8, measure_int=2, ctx=gpu_ctx, checkpoint=f, checkpoint_int=4)
    b, obs = GDR.run_density(pg, chi, dt, n, w=8, measure_int=2, ctx=gpu_ctx, checkpoint=f)
    assert all(np.array_equal(a, c) for a, c in zip(b.rho.sites(), b_ref.rho.sites()))
    assert len(obs) == len(obs_ref)
    for (t, s, m), (tr, sr, mr) in zip(obs, obs_ref):
        assert t == tr and np.array_equal(s, sr) and np.array_equal(m, mr)
