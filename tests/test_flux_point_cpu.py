"""The flux kernels' point functions (canard_b200/csrc/kernels.cuh), compiled
for the host and checked against the reference's point formulas in FP64: the
viscous stresses and heat flux of calc_viscous_shear_stress
(src/mo_physics.f90:245-299) and the flux components of calc_fluxes
(src/mo_physics.f90:319-382). FP32: flux_visc_values, the point of
k_flux_visc_pairs, with the conserved values formed from the primitives as
the FP32-mixed step path does. FP64: visc_point and flux_point as
k_flux_visc<double> (state preloaded) and k_flux (the phase API) call them.
Viscous and inviscid points, with a moving frame. No GPU: the harness calls
no CUDA API."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else None)


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if NVCC is None:
        pytest.skip("nvcc not found")
    exe = str(tmp_path_factory.mktemp("fluxpt") / "flux_point_check")
    subprocess.run([NVCC, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "canard_b200", "csrc"),
                    os.path.join(ROOT, "tests", "flux_point_check.cu"), "-o", exe], check=True, timeout=600)
    return exe


def run_harness(exe, a, visc, um, mode=0):
    """mode 0: FP32 point function on a[:, :28]; 1: FP64 fused form; 2: FP64
    phase form, both on a[:, :33] (the conserved values in a[:, 28:33])."""
    dt = np.float32 if mode == 0 else np.float64
    cols = 28 if mode == 0 else 33
    head = np.array([mode, a.shape[0], int(visc)], np.int32).tobytes() + np.asarray(um, np.float64).tobytes()
    r = subprocess.run([exe], input=head + np.ascontiguousarray(a[:, :cols], dt).tobytes(), capture_output=True,
                       timeout=60)
    assert r.returncode == 0, r.returncode
    return np.frombuffer(r.stdout, dt).reshape(a.shape[0], 16)


def reference_point(a, visc, um, qa=None):
    """FP64 statement of the reference's point formulas. a[:, 3f + d]: the
    derivative along direction d of variable f (u, v, w, T); a[:, 12 + 3d + c]:
    metric term c of direction d (xim, etm, zem); then mu, yaco, p, 1/rho, u,
    v, w. qa: the conserved values, else formed from the primitives."""
    g = a[:, :12]
    mt = a[:, 12:21].reshape(-1, 3, 3)
    mu, yaco, p, rinv, u, v, w = (a[:, 21 + k] for k in range(7))
    n = a.shape[0]
    tau = np.zeros((n, 3, 3))
    h = np.zeros((n, 3))
    if visc:
        def comb(f, c):
            return mt[:, 0, c] * g[:, 3 * f] + mt[:, 1, c] * g[:, 3 * f + 1] + mt[:, 2, c] * g[:, 3 * f + 2]
        txx, hzz, tzx = comb(0, 0), comb(0, 1), comb(0, 2)
        txy, tyy, hxx = comb(1, 0), comb(1, 1), comb(1, 2)
        hyy, tyz, tzz = comb(2, 0), comb(2, 1), comb(2, 2)
        s = [comb(3, c) for c in range(3)]
        rr1 = mu * yaco
        rr2 = rr1 / (0.4 * 0.71)
        d5 = 2.0 / 3.0 * (txx + tyy + tzz)
        txx, tyy, tzz = rr1 * (2 * txx - d5), rr1 * (2 * tyy - d5), rr1 * (2 * tzz - d5)
        txy, tyz, tzx = rr1 * (txy + hzz), rr1 * (tyz + hxx), rr1 * (tzx + hyy)
        h[:, 0] = rr2 * s[0] + u * txx + v * txy + w * tzx
        h[:, 1] = rr2 * s[1] + u * txy + v * tyy + w * tyz
        h[:, 2] = rr2 * s[2] + u * tzx + v * tyz + w * tzz
        tau[:, 0] = np.stack([txx, txy, tzx], 1)
        tau[:, 1] = np.stack([txy, tyy, tyz], 1)
        tau[:, 2] = np.stack([tzx, tyz, tzz], 1)
    if qa is None:
        rho = 1.0 / rinv
        qa = np.stack([rho, rho * u, rho * v, rho * w, p / 0.4 + 0.5 * rho * (u * u + v * v + w * w)], 1)
    vel = np.stack([u + um[0], v + um[1], w + um[2]], 1)
    ss = np.einsum("ndc,nc->nd", mt, vel)
    out = np.zeros((n, 16))
    out[:, 0:3] = qa[:, :1] * ss
    for c in range(3):
        for d in range(3):
            out[:, 3 * (c + 1) + d] = qa[:, c + 1] * ss[:, d] + mt[:, d, c] * p \
                - np.einsum("nk,nk->n", mt[:, d, :], tau[:, c, :])
    de5 = qa[:, 4] + p
    for d in range(3):
        out[:, 12 + d] = de5 * ss[:, d] - p * (mt[:, d, :] @ np.asarray(um, float)) \
            - np.einsum("nk,nk->n", mt[:, d, :], h)
    out[:, 15] = de5
    return out


def point_inputs(n, seed):
    rng = np.random.default_rng(seed)
    a = np.empty((n, 28))
    a[:, :12] = rng.standard_normal((n, 12))
    a[:, 12:21] = (np.eye(3).ravel() + 0.2 * rng.standard_normal((n, 9)))
    a[:, 21] = rng.uniform(0.05, 0.2, n)     # mu: stresses of the order of the pressure terms
    a[:, 22] = rng.uniform(0.5, 2.0, n)      # yaco
    a[:, 23] = rng.uniform(0.5, 1.0, n)      # p
    a[:, 24] = rng.uniform(0.5, 2.0, n)      # 1/rho
    a[:, 25:28] = 0.3 * rng.standard_normal((n, 3))
    return a.astype(np.float32).astype(np.float64)


def conserved(a):
    """The five conserved values of the points' primitives (for the FP64 forms,
    which read the state)."""
    rho = 1.0 / a[:, 24]
    u, v, w, p = a[:, 25], a[:, 26], a[:, 27], a[:, 23]
    return np.stack([rho, rho * u, rho * v, rho * w, p / 0.4 + 0.5 * rho * (u * u + v * v + w * w)], 1)


@pytest.mark.parametrize("visc", [1, 0])
def test_flux_point_matches_reference_formulas(harness, visc):
    um = (0.1, -0.05, 0.02)
    a = point_inputs(4096, seed=5 + visc)
    got = run_harness(harness, a, visc, um).astype(np.float64)
    ref = reference_point(a, visc, um)
    for k in range(16):
        err = np.linalg.norm(got[:, k] - ref[:, k]) / np.linalg.norm(ref[:, k])
        assert err <= 1e-6, (k, err)
    if visc:
        # the viscous terms are not negligible in these inputs
        assert np.linalg.norm(ref - reference_point(a, 0, um)) > 0.1 * np.linalg.norm(ref)


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("visc", [1, 0])
def test_fp64_flux_point_matches_reference_formulas(harness, visc, mode):
    um = (0.1, -0.05, 0.02)
    a = point_inputs(4096, seed=11 + visc)
    qa = conserved(a)
    got = run_harness(harness, np.concatenate([a, qa], 1), visc, um, mode)
    ref = reference_point(a, visc, um, qa)
    for k in range(16):
        err = np.linalg.norm(got[:, k] - ref[:, k]) / np.linalg.norm(ref[:, k])
        assert err <= 1e-14, (k, err)
