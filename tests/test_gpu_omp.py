"""The OpenMP integrator's semantics on the device (MI_SEM_OMP, IntegratorZarrOMP.c:1709-1847):
the IntegrationCore sums, a nonzero sum divided by the bin's whole area, bins of the bin mask
NaN, the lineout as the mean of each row's nonzero, non-NaN bins -- for every encoding,
against the FP64 oracle and against the compiled reference integrator's own sums."""
import numpy as np
import pytest
import torch

import oracle
from conftest import MAPPER_CASES, load_mapper_case, rel_err
from midas_b200 import _lib as L
from midas_b200.bin_io import from_arrays
from midas_b200.kernels import CakePlan

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", MAPPER_CASES)
@pytest.mark.parametrize("mode", ["bilinear", "gradient"])
@pytest.mark.parametrize("enc", ["runs", "csr", "mma", "mmad"])
def test_omp_semantics_matches_oracle_and_reference_sums(cuda, tag, mode, enc):
    g = load_mapper_case(tag)
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    nb = n_r * n_eta
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode=mode, semantics="omp",
                    bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding=enc)
    mask = np.random.default_rng(7).random(nb) < 0.05
    plan.set_bin_mask(mask)
    plan.set_dark(g["dark"].astype(np.float32))
    rng = np.random.default_rng(1)
    frames = np.concatenate([np.rint(g["image"])[None].clip(0, 65535),
                             rng.integers(0, 30000, size=(4, g["nz"], g["ny"]))]).astype(np.uint16)
    ck, aw, sm = plan.integrate(torch.from_numpy(frames).to(cuda))
    ck, aw, sm = ck.cpu().numpy().reshape(len(frames), -1), aw.cpu().numpy(), sm.cpu().numpy()
    assert plan.status() == 0
    a_in = oracle.area_in(g["records"], g["nmap"], nb, g["ny"], g["nz"])
    for f in range(len(frames)):
        assert np.isnan(ck[f][mask]).all() and not np.isnan(ck[f][~mask]).any()
        sub = frames[f].astype(np.float32) - g["dark"].astype(np.float32)
        ref, _ = oracle.integrate(g["records"], g["nmap"], nb, g["ny"], g["nz"], sub.astype(np.float64), mode=mode,
                                  semantics="omp", bc_y=g["bc_y"], bc_z=g["bc_z"])
        assert rel_err(ck[f][~mask], ref[~mask])[0] <= 1e-6
        ref = np.where(mask, np.nan, ref)
        raw, rsm = oracle.profile_omp(ref, a_in, n_r, n_eta)
        assert rel_err(aw[f], raw)[0] <= 1e-6 and rel_err(sm[f], rsm)[0] <= 1e-6
    if enc in ("runs", "csr"):
        # the fixture's own float image against integration_apply_map's sums and norms
        sums, norms = g[f"ic_sums_{mode}"], g[f"ic_norms_{mode}"]
        want = np.where(sums != 0, sums / np.where(norms != 0, norms, 1.0), 0.0)
        img = torch.from_numpy(g["image"].astype(np.float32)[None]).to(cuda)
        c0, _, _ = plan.integrate(img)
        c0 = c0.cpu().numpy().reshape(-1)
        assert rel_err(c0[~mask], want[~mask])[0] <= 1e-6
    plan.close()


def test_omp_semantics_needs_the_cake_for_its_lineouts(cuda):
    g = load_mapper_case("m2")
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    plan = CakePlan(from_arrays(g["records"], g["nmap"]), n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"],
                    n_pixels_z=g["nz"], mode="gradient", semantics="omp", bc_y=g["bc_y"], bc_z=g["bc_z"],
                    device=cuda)
    frames = torch.zeros((1, g["nz"], g["ny"]), dtype=torch.uint16, device=cuda)
    aw = torch.empty((1, n_r), dtype=torch.float64, device=cuda)
    rc = L.lib().mi_integrate_batch(plan._h, frames.data_ptr(), L.DT_U16, 1, g["ny"] * g["nz"], None,
                                    aw.data_ptr(), None, L.stream_ptr())
    assert rc == L.MI_E_ARG and b"cake" in L.lib().mi_last_error()
    with pytest.raises(L.MidasError):
        CakePlan(from_arrays(g["records"], g["nmap"]), n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"],
                 n_pixels_z=g["nz"], mode="floor", semantics="omp", device=cuda)
