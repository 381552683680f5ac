"""GPU clutter filter and filtered-PD pipeline against the complex128 oracle (reference test_gpu_clutter.py)."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import clutter as oc
from oracle import das
from rcabeam_b200 import _lib, gpu_clutter, pipeline
from rcabeam_b200.sim import RCAGeometry
from tests._cases import oracle_inputs, rel_l2

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    yield
    assert _lib.device_error() == 0


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("shape", [(7,), (3, 7), (19, 6), (2, 4, 6), (2, 1), (16385, 4)])
@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_gram_basis_and_filter_parity(shape, dtype):
    rng = np.random.default_rng(8)
    host = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(dtype)
    iq = _dev(host)
    original = iq.clone()
    timings = {}
    values, basis = gpu_clutter.temporal_basis(iq, timings=timings)
    assert timings["matrix_seconds"] >= 0 and timings["decomposition_seconds"] >= 0
    expected_values, _ = oc.temporal_basis(host)
    np.testing.assert_allclose(values.cpu().numpy(), expected_values, rtol=1e-7, atol=1e-7)
    np.testing.assert_allclose((basis.conj().T @ basis).cpu().numpy(), np.eye(shape[-1]), atol=2e-14)
    end = min(3, shape[-1])
    actual = gpu_clutter.apply_temporal_filter(iq, basis, rank_start=0, rank_stop=end)
    expected = oc.svd_clutter_filter(host, rank_start=0, rank_stop=end)
    assert actual.dtype == iq.dtype and tuple(actual.shape) == shape
    assert torch.equal(iq, original)
    np.testing.assert_allclose(actual.cpu().numpy(), expected, rtol=2e-6, atol=2e-6)
    np.testing.assert_allclose(gpu_clutter.svd_clutter_filter(iq, rank_start=0).cpu().numpy(), host, atol=1e-6)
    assert not gpu_clutter.apply_temporal_filter(iq, basis, rank_start=shape[-1]).cpu().numpy().any()


def test_known_spectrum_golden():
    c = np.load(GOLDEN / "clutter.npz")
    iq = _dev(c["spectrum_matrix"].reshape(3, 6, 6))
    values, basis = gpu_clutter.temporal_basis(iq)
    np.testing.assert_allclose(values.cpu().numpy(), c["spectrum_values"], rtol=2e-6)
    out = gpu_clutter.svd_clutter_filter(iq, rank_start=1, rank_stop=4)
    np.testing.assert_allclose(out.cpu().numpy(), c["spectrum_gram_filtered"], rtol=2e-5, atol=2e-6)


def test_tissue_clutter_rank3_golden():
    """Strong rank-3 clutter removed: filtered IQ and power vs the reference (complex64 output)."""
    c = np.load(GOLDEN / "clutter.npz")
    iq = _dev(c["tissue_iq"])
    out = gpu_clutter.svd_clutter_filter(iq, rank_start=3).cpu().numpy()
    ref = c["tissue_gram_filtered"]
    assert rel_l2(out, ref) < 1e-6
    _, basis = gpu_clutter.temporal_basis(iq)
    power = gpu_clutter.filtered_power(iq, basis, rank_start=3).cpu().numpy()
    _, b64 = oc.temporal_basis(c["tissue_iq"], method="gram")
    np.testing.assert_allclose(power, oc.filtered_power(c["tissue_iq"], b64, 3), rtol=1e-9)


@pytest.mark.parametrize("start,stop,modes", [(2, 200, 2), (2, 5, 3), (0, 200, 0), (0, 0, 0), (200, 200, 0)])
def test_smaller_projector_and_power(start, stop, modes):
    rng = np.random.default_rng(12)
    host = rng.normal(size=(17, 200)) + 1j * rng.normal(size=(17, 200))
    iq = _dev(host)
    basis = torch.eye(200, dtype=torch.complex128, device="cuda")
    expected = np.zeros_like(host)
    expected[:, start:stop] = host[:, start:stop]
    actual = gpu_clutter.apply_temporal_filter(iq, basis, rank_start=start, rank_stop=stop)
    power = gpu_clutter.filtered_power(iq, basis, rank_start=start, rank_stop=stop)
    np.testing.assert_allclose(actual.cpu().numpy(), expected, atol=1e-13)
    np.testing.assert_allclose(power.cpu().numpy(), np.mean(np.abs(expected) ** 2, axis=-1), atol=1e-13)
    _, subtract = gpu_clutter._filter_vectors(basis, 200, start, stop)
    assert subtract == (stop - start > 200 - (stop - start))


def test_shared_rc_cr_basis_and_weak_band():
    rng = np.random.default_rng(19)
    left, _ = np.linalg.qr(rng.normal(size=(24, 6)) + 1j * rng.normal(size=(24, 6)))
    right, _ = np.linalg.qr(rng.normal(size=(6, 6)) + 1j * rng.normal(size=(6, 6)))
    host = (left * np.array([1e4, 2, 1, 0.3, 0.1, 0.01])) @ right.conj().T
    pair = (_dev(host[:12].reshape(3, 4, 6)), _dev(host[12:].reshape(2, 6, 6)))
    actual = gpu_clutter.svd_clutter_filter(pair, rank_start=1, rank_stop=5)
    expected = oc.svd_clutter_filter(host, rank_start=1, rank_stop=5)
    joined = np.concatenate([a.cpu().numpy().reshape(-1, 6) for a in actual])
    assert rel_l2(joined, expected) < 1e-5


@pytest.mark.parametrize("amplitude", [1e38, 1e-40])
def test_scaled_gram_avoids_overflow_and_underflow(amplitude):
    iq = torch.full((64, 8), complex(amplitude, amplitude), dtype=torch.complex64, device="cuda")
    diagnostics = {}
    values, basis = gpu_clutter.temporal_basis(iq, diagnostics=diagnostics)
    expected, _ = oc.temporal_basis(iq.cpu().numpy())
    assert values.dtype == torch.float64
    np.testing.assert_allclose(float(values[0]), expected[0], rtol=2e-6)
    assert diagnostics["input_scale"] == float(iq.real[0, 0])
    power = gpu_clutter.filtered_power(iq, basis, rank_start=0)
    np.testing.assert_allclose(power.cpu().numpy(), np.full(64, 2 * float(iq.real[0, 0]) ** 2), rtol=1e-6)


def test_residual_power_does_not_subtract_large_energies():
    basis = np.array([[1, 1, 1, 1], [1, -1, 1, -1], [1, 1, -1, -1], [1, -1, -1, 1]], complex).T / 2
    host = (1e8 * basis[:, 0] + basis[:, 1])[None, :]
    actual = gpu_clutter.filtered_power(_dev(host), _dev(basis), rank_start=1)
    np.testing.assert_allclose(actual.cpu().numpy(), [0.25], atol=1e-14)


def test_negative_eigenvalue_policy(monkeypatch):
    decompose = gpu_clutter.Gram.decompose

    def broken(self):
        decompose(self)
        self.eigenvalues[0] = -1.0

    monkeypatch.setattr(gpu_clutter.Gram, "decompose", broken)
    with pytest.raises(np.linalg.LinAlgError, match="negative"):
        gpu_clutter.temporal_basis(torch.ones((3, 4), dtype=torch.complex128, device="cuda"))


def test_invalid_inputs():
    iq = torch.ones((3, 4), dtype=torch.complex64, device="cuda")
    for bad in ((), np.ones((2, 4), complex), torch.ones((2, 4), device="cuda"),
                torch.empty((0, 4), dtype=torch.complex64, device="cuda"),
                torch.tensor([complex(np.nan, 1)], dtype=torch.complex64, device="cuda")):
        with pytest.raises(ValueError):
            gpu_clutter.temporal_basis(bad)
    with pytest.raises(ValueError, match="frame count"):
        gpu_clutter.temporal_basis((iq, torch.ones((3, 5), dtype=torch.complex64, device="cuda")))
    with pytest.raises(ValueError, match="Precision"):
        gpu_clutter.temporal_basis(iq, precision="float32")
    for basis in (np.eye(4), torch.eye(3, dtype=torch.complex128, device="cuda"),
                  torch.ones((4, 4), dtype=torch.complex128, device="cuda")):
        with pytest.raises(ValueError, match="Basis"):
            gpu_clutter.apply_temporal_filter(iq, basis, rank_start=0)
    for start, stop in ((True, None), (-1, 4), (0, 5), (3, 2)):
        with pytest.raises(ValueError, match=r"Rank|rank"):
            gpu_clutter.svd_clutter_filter(iq, rank_start=start, rank_stop=stop)


def test_power_doppler():
    rng = np.random.default_rng(4)
    x = (rng.normal(size=(5, 7, 33)) + 1j * rng.normal(size=(5, 7, 33))).astype(np.complex64)
    np.testing.assert_allclose(gpu_clutter.power_doppler(x), das.power_doppler(x), rtol=1e-6)
    np.testing.assert_allclose(gpu_clutter.power_doppler(_dev(x)).cpu().numpy(), das.power_doppler(x), rtol=1e-6)


def _scene(frames=24, seed=5):
    """Small RCA scene: slowly moving strong tissue speckle + weak random blood + noise."""
    el = (np.arange(16) - 7.5) * 0.2e-3
    geom = RCAGeometry(el, el, c=1540.0, fs=20e6, f_demod=15e6, fnumber=None)
    angles = np.deg2rad(np.linspace(-8, 8, 3))
    rng = np.random.default_rng(seed)
    ns, t0 = 160, 4e-6
    t = t0 + np.arange(ns) / 20e6
    rc = np.zeros((ns, 16, 3, frames), np.complex128)
    cr = np.zeros_like(rc)
    pts = np.column_stack([rng.uniform(-1.5e-3, 1.5e-3, 60), rng.uniform(4e-3, 6e-3, 60),
                           rng.uniform(-1.5e-3, 1.5e-3, 60)])
    amp = rng.normal(size=60) + 1j * rng.normal(size=60)
    amp[40:] *= 0.01
    for f in range(frames):
        shift = np.zeros(3)
        shift[1] = 2e-6 * f
        moved = pts + shift
        moved[40:, 0] += 1e-5 * f * rng.normal()
        for cfg, out in (("RC", rc), ("CR", cr)):
            elx = el
            for p, a in zip(moved, amp):
                v, u = (p[0], p[2]) if cfg == "RC" else (p[2], p[0])
                recv = np.sqrt(p[1] ** 2 + (v - elx) ** 2) / 1540.0
                for m, th in enumerate(angles):
                    tau = (p[1] * np.cos(th) + u * np.sin(th)) / 1540.0 + recv
                    env = np.exp(-(((t[:, None] - tau[None, :]) / 0.15e-6) ** 2))
                    out[:, :, m, f] += a * env * np.exp(-2j * np.pi * 15e6 * tau)[None, :]
    noise = 1e-3 * (rng.normal(size=rc.shape) + 1j * rng.normal(size=rc.shape))
    grid = (np.linspace(-1e-3, 1e-3, 6), np.linspace(4.2e-3, 5.8e-3, 10), np.linspace(-1e-3, 1e-3, 5))
    return (rc + noise).astype(np.complex64), (cr + noise).astype(np.complex64), angles, t0, grid, geom


def test_filtered_pipeline_matches_fp64_oracle():
    """DAS -> Gram -> EVD -> filtered power vs the float64 oracle chain: relative L2 <= 1e-4 (target bar)."""
    rc, cr, angles, t0, grid, geom = _scene()
    o = oracle_inputs(angles, t0, grid, geom)
    iq = das.opw_iq(rc, cr, o["scan"], o["xe"], o["ye"], o["angles"], o["starts"], o["c"], o["fs"], o["fd"],
                    o["fnumber"])
    _, basis = oc.temporal_basis(iq, method="gram")
    expected = oc.filtered_power(iq, basis, 3).reshape(6, 10, 5)
    plan = pipeline.FilteredOpw(rc.shape, angles, t0, grid, geom, rank_start=3)
    got = plan.run(_dev(rc), _dev(cr))
    plan.check()
    assert rel_l2(got.cpu().numpy(), expected) < 1e-4
    host = plan.run_host(torch.from_numpy(rc).pin_memory(), torch.from_numpy(cr).pin_memory())
    plan.check()
    assert rel_l2(host.numpy().reshape(6, 10, 5), expected) < 1e-4


@pytest.mark.parametrize("storage,precision,domain,deterministic", [("float32", "complex128", "beamformed", False),
                                                                    ("bf16x2", "bf16x3", "beamformed", False),
                                                                    ("bf16x2", "bf16x3", "beamformed", True),
                                                                    ("bf16x2", "bf16x3", "channel", False)])
def test_host_sequence_matches_single_runs(storage, precision, domain, deterministic):
    """run_host_sequence (uploads overlapping the previous ensemble's reconstruction) returns, for
    three different ensembles in a row, the powers of separate runs.  The SIMT path is deterministic;
    by default the tensor-core DAS starts each item's channel walk where the other CTAs are, so its
    float32 sums run in a timing-dependent order (~1e-7 of the IQ), which removing the 100x stronger
    tissue signal amplifies in the filtered power: 5e-5, under the 1e-4 bar of the filtered pipeline.
    With ``deterministic=True`` every tile walks its channels from the same slot, so only the
    interleaving of the builder warps' steps stays timing dependent: 2e-6 to 1.1e-5 measured."""
    scenes = [_scene(seed=s) for s in (5, 6, 7)]
    _, _, angles, t0, grid, geom = scenes[0]
    plan = pipeline.FilteredOpw(scenes[0][0].shape, angles, t0, grid, geom, rank_start=3, precision=precision,
                                iq_storage=storage, domain=domain, deterministic=deterministic)
    single = [plan.run(_dev(rc), _dev(cr)).cpu().numpy().ravel() for rc, cr, *_ in scenes]
    pairs = [(torch.from_numpy(rc).pin_memory(), torch.from_numpy(cr).pin_memory()) for rc, cr, *_ in scenes]
    outs = plan.run_host_sequence(pairs)
    plan.check()
    assert len(outs) == 3
    tol = 1e-12 if storage == "float32" else (2.5e-5 if deterministic else 6e-5)
    for got, want in zip(outs, single):
        assert rel_l2(got.numpy(), want) <= tol
    with pytest.raises(ValueError, match="one output"):
        plan.run_host_sequence(pairs, outputs=outs[:2])


@pytest.mark.parametrize("n", [1, 2, 7, 4096, 1_000_003])
@pytest.mark.parametrize("offset", [0, 1])
def test_scale_max_abs_matches_torch(n, offset):
    """rcabeam_clutter_scale_device on complex64 (vectorized path for 16-byte aligned data, the
    scalar path for an 8-byte offset) equals max |re|, |im| exactly, odd lengths included."""
    g = torch.Generator(device="cuda").manual_seed(n)
    buf = torch.randn((n + 1) * 2, generator=g, device="cuda", dtype=torch.float32)
    buf[2 * offset + 2 * (n - 1) + 1] = 7.5  # the largest component sits in the last sample
    x = torch.view_as_complex(buf.view(-1, 2))[offset:offset + n]
    scale = torch.zeros(1, dtype=torch.float64, device="cuda")
    _lib.call("rcabeam_clutter_scale_device", x.data_ptr(), n, 0, scale.data_ptr())
    want = torch.view_as_real(x).abs().max().double()
    assert float(scale.item()) == float(want.item()) == 7.5


@pytest.mark.parametrize("rows,nt", [(1, 2), (31, 8), (33, 64), (1000, 128), (70001, 200), (257, 256), (65, 258),
                                     (4097, 400), (40, 512), (5, 199)])
@pytest.mark.parametrize("k,mode", [(3, 1), (3, 3), (1, 0), (4, 2), (2, 1)])
@pytest.mark.parametrize("offset", [0, 1])
def test_projection_rows_match_float64(rows, nt, k, mode, offset):
    """rcabeam_project_device on complex64 rows (ragged row counts, odd and even frame counts,
    aligned and 8-byte offset rows, every mode) against float64 NumPy: power to 1e-11
    relative, written rows to float32 rounding."""
    if k > nt:
        pytest.skip("k temporal vectors need k <= nt frames")
    rng = np.random.default_rng(rows + nt + k)
    host = (rng.normal(size=(rows, nt)) + 1j * rng.normal(size=(rows, nt))).astype(np.complex64)
    host[:, :] += 50 * np.exp(2j * np.pi * 0.01 * np.arange(nt))  # a strong common component
    q, _ = np.linalg.qr(rng.normal(size=(nt, k)) + 1j * rng.normal(size=(nt, k)))
    flat = torch.zeros(rows * nt + 1, dtype=torch.complex64, device="cuda")
    iq = flat[offset:offset + rows * nt]
    iq.copy_(torch.from_numpy(host.ravel()))
    vec = _dev(np.asfortranarray(q).ravel(order="F"))
    out = torch.zeros(rows * nt, dtype=torch.complex64, device="cuda") if mode & 2 else None
    power = torch.zeros(rows, dtype=torch.float64, device="cuda")
    flags = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("rcabeam_project_device", iq.data_ptr(), None if out is None else out.data_ptr(), power.data_ptr(),
              rows, nt, 0, vec.data_ptr(), k, mode, flags.data_ptr())
    assert int(flags.item()) == 0
    x = host.astype(np.complex128)
    y = x @ q
    part = y @ q.conj().T
    resid = x - part if mode & 1 else part
    want = (np.sum(np.abs(resid) ** 2, axis=1) if mode & 1 else np.sum(np.abs(y) ** 2, axis=1)) / nt
    got = power.cpu().numpy()
    scale = np.mean(np.abs(x) ** 2)  # a residual can be exactly zero (k = nt): rounding is relative to |x|^2
    np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-12 * max(want.max(), scale))
    if out is not None:
        np.testing.assert_allclose(out.cpu().numpy().reshape(rows, nt), resid, rtol=0,
                                   atol=2e-6 * np.abs(resid).max() + 1e-6)


@pytest.mark.parametrize("rows,nt,m", [(1, 8, 1), (1000, 64, 16), (20001, 200, 16), (333, 400, 5)])
def test_ritz_matrix_is_float64_projected_gram(rows, nt, m):
    """rcabeam_ritz_matrix_device forms (X V)^H (X V) in float64 (complex64 rows, column-major)."""
    rng = np.random.default_rng(rows + m)
    host = (rng.normal(size=(rows, nt)) + 1j * rng.normal(size=(rows, nt))).astype(np.complex64)
    v = rng.normal(size=(m, nt)) + 1j * rng.normal(size=(m, nt))  # vector c in row c
    iq, vec = _dev(host), _dev(v)
    h = torch.empty(m * m, dtype=torch.complex128, device="cuda")
    _lib.call("rcabeam_ritz_matrix_device", iq.data_ptr(), rows, nt, vec.data_ptr(), m, h.data_ptr())
    y = host.astype(np.complex128) @ v.T
    want = y.conj().T @ y
    got = h.cpu().numpy().reshape(m, m).T  # column-major storage
    np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-11 * np.abs(want).max())


def test_ritz_refinement_is_the_float64_ritz_step():
    """The Rayleigh-Ritz step on the 3xBF16 Gram's 16 leading vectors equals a complex128 Ritz step
    over the same subspace, and its leading span is no farther from the float64 Gram's than the
    unrefined vectors (the step removes only the error that lies inside the 16-vector subspace)."""
    gen = torch.Generator(device="cuda").manual_seed(4)
    from rcabeam_b200 import scenes

    iq = scenes.clutter_casorati(200_000, 64, generator=gen, device="cuda")
    _, b64 = gpu_clutter.temporal_basis(iq)
    _, b16 = gpu_clutter.temporal_basis(iq, precision="bf16x3")
    m, k = 16, 3
    basis = b16[:, :m].transpose(0, 1).contiguous()  # vector c in row c
    h = gpu_clutter.Gram(m, iq.device)
    _lib.call("rcabeam_ritz_matrix_device", iq.data_ptr(), iq.shape[0], 64, basis.data_ptr(), m, h.matrix.data_ptr())
    h.decompose()
    u = torch.view_as_complex(h.matrix.view(m, m, 2))[m - k:]  # eigenvector j in row j, ascending
    refined = (u @ basis).transpose(0, 1)

    y = iq.to(torch.complex128) @ basis.transpose(0, 1)
    _, w = torch.linalg.eigh(y.conj().transpose(0, 1) @ y)
    want = basis.transpose(0, 1) @ w[:, m - k:]
    proj = lambda b: b @ b.conj().transpose(0, 1)  # noqa: E731
    assert torch.linalg.matrix_norm(proj(refined) - proj(want)).item() < 1e-9

    p64 = proj(b64[:, :k])
    err = lambda b: torch.linalg.matrix_norm(proj(b) - p64).item()  # noqa: E731
    assert err(refined) <= err(b16[:, :k]) * (1 + 1e-6)


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
@pytest.mark.parametrize("k,nt", [(3, 64), (3, 400), (6, 64)])
def test_projection_flags_non_finite_input_and_power(dtype, k, nt):
    """The projection's flags word: bit 0 for a NaN or infinite input component (both the
    persistent kernel, k <= 4, and the general one), bit 1 for an overflowing power."""
    rows = 1000
    gen = torch.Generator(device="cuda").manual_seed(k + nt)
    x = torch.randn((rows, nt), dtype=dtype, device="cuda", generator=gen)
    q, _ = torch.linalg.qr(torch.randn((nt, k), dtype=torch.complex128, device="cuda", generator=gen))
    vec = q.transpose(0, 1).contiguous()  # column-major (nt x k)
    power = torch.empty(rows, dtype=torch.float64, device="cuda")

    def flags_of(a):
        flags = torch.zeros(1, dtype=torch.int32, device="cuda")
        _lib.call("rcabeam_project_device", a.data_ptr(), None, power.data_ptr(), rows, nt,
                  int(a.dtype == torch.complex128), vec.data_ptr(), k, 1, flags.data_ptr())
        return int(flags.item())

    assert flags_of(x) == 0
    for bad in (complex(float("nan"), 0.0), complex(0.0, float("inf"))):
        y = x.clone()
        y[517, nt // 3] = bad
        assert flags_of(y) & 1
    if dtype == torch.complex128:
        assert flags_of(x * 1e200) == 2  # finite input, |x|^2 overflows


def test_filtered_power_and_basis_reject_non_finite_input():
    """filtered_power and temporal_basis raise the reference's ValueError for NaN / infinite IQ
    (gpu_clutter.py:36-37) from the projection flags and the Casorati scale."""
    iq = torch.randn((300, 16), dtype=torch.complex64, device="cuda")
    _, basis = gpu_clutter.temporal_basis(iq)
    for bad in (complex(float("nan"), 1.0), complex(float("-inf"), 0.0)):
        y = iq.clone()
        y[123, 7] = bad
        with pytest.raises(ValueError, match="finite"):
            gpu_clutter.filtered_power(y, basis, rank_start=2)
        with pytest.raises(ValueError, match="finite"):
            gpu_clutter.filtered_power(y, basis, rank_start=2, rank_stop=2)
        for precision in ("complex128", "bf16x3"):
            with pytest.raises(ValueError, match="finite"):
                gpu_clutter.temporal_basis(y, precision=precision)


def _project_case(rows, frames, k, seed):
    rng = np.random.default_rng(seed)
    x = (rng.normal(size=(rows, frames)) + 1j * rng.normal(size=(rows, frames))).astype(np.complex64)
    x[:, :] *= np.exp(rng.normal(size=(rows, 1)))  # row scales over a few orders of magnitude
    q, _ = np.linalg.qr(rng.normal(size=(frames, k)) + 1j * rng.normal(size=(frames, k)))
    return x, q  # q: (frames, k) orthonormal columns


@pytest.mark.parametrize("frames", [33, 37, 64, 201, 256, 257, 400, 511, 512])
@pytest.mark.parametrize("k", [1, 3, 4])
def test_projection_residual_against_float64(frames, k):
    """rcabeam_project_device with the smaller projector subtracted (the float64
    tensor-core form for complex64 rows, k <= 4, 33-512 frames): power (mode 1) and
    filtered IQ (mode 3) against x - (x V) V^H in complex128 (gpu_clutter.py:212-273),
    on 1001 rows (not a multiple of the 8-row tiles) and frame counts off the 4-frame
    tiles."""
    x, v = _project_case(1001, frames, k, seed=frames * 10 + k)
    xd = x.astype(np.complex128)
    resid = xd - (xd @ v) @ v.conj().T
    want_pw = np.sum(np.abs(resid) ** 2, axis=1) / frames
    dx = _dev(x)
    vec = _dev(np.ascontiguousarray(v.T))  # (k, frames): vector c in row c
    power = torch.empty(x.shape[0], dtype=torch.float64, device="cuda")
    flags = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("rcabeam_project_device", dx.data_ptr(), None, power.data_ptr(), x.shape[0], frames, 0, vec.data_ptr(),
              k, 1, flags.data_ptr())
    np.testing.assert_allclose(power.cpu().numpy(), want_pw, rtol=1e-12, atol=0)
    out = torch.empty_like(dx)
    _lib.call("rcabeam_project_device", dx.data_ptr(), out.data_ptr(), None, x.shape[0], frames, 0, vec.data_ptr(),
              k, 3, flags.data_ptr())
    got = out.cpu().numpy()
    # complex64 rounding of the residual (relative to each row's magnitude)
    scale = np.abs(xd).max(axis=1, keepdims=True)
    assert np.max(np.abs(got - resid) / scale) <= 2e-7
    assert int(flags.item()) == 0


def test_projection_flags_non_finite_rows():
    """A non-finite input component sets flag bit 0 and its non-finite power bit 1."""
    x, v = _project_case(64, 200, 3, seed=5)
    x[17, 101] = np.nan
    dx = _dev(x)
    vec = _dev(np.ascontiguousarray(v.T))
    power = torch.empty(x.shape[0], dtype=torch.float64, device="cuda")
    flags = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("rcabeam_project_device", dx.data_ptr(), None, power.data_ptr(), x.shape[0], 200, 0, vec.data_ptr(),
              3, 1, flags.data_ptr())
    assert int(flags.item()) == 3
    pw = power.cpu().numpy()
    assert not np.isfinite(pw[17]) and np.isfinite(np.delete(pw, 17)).all()
