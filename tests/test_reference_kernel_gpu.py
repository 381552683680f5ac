"""GPU parity and timing of the B200 library against the reference's own CUDA kernels.

``oracle/build_ref.py`` compiles the reference's ``core.cu`` + ``ensemble.cu``
unchanged for sm_100a into ``oracle/_ref/librcabeam_ref.so``.  Both libraries
export the same C names; each is loaded privately through ctypes and called
with the same device buffers.

* Packing is a pure transpose (and an FP16 round-to-nearest): bit-identical.
* Every ensemble method and every per-frame entry point agrees with the
  reference kernels within 5e-4 relative L2 -- the reference's own ensemble
  tolerance (tests/test_ensemble.py) -- and the B200 library is at least as
  close to the float64 oracle (it forms delays in float64; the reference in
  float32).
* At the full workload the test times the reference's binding loop (16384-voxel
  tiles, src/rcabeam/bindings/python.cpp:553-565) against the B200 paths with
  CUDA events and prints the table (``-s`` shows it).
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import das, methods
from rcabeam_b200 import _cuda_impl, _lib
from rcabeam_b200.sim import RCAGeometry, scan_coords
from tests._cases import oracle_inputs, random_case, rel_l2

pytestmark = pytest.mark.gpu

REF_PATH = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "librcabeam_ref.so"
TOL = 5e-4


@pytest.fixture(scope="module")
def ref():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    if not REF_PATH.exists():
        pytest.skip("reference CUDA library not built (python oracle/build_ref.py)")
    handle = ctypes.CDLL(str(REF_PATH))
    # The reference exports the names of its own header only; bind those.
    for name in (n for n in _lib.SIGNATURES if hasattr(handle, n)):
        fn = getattr(handle, name)
        fn.argtypes = _lib.SIGNATURES[name]
        fn.restype = ctypes.c_int
    return handle


@pytest.fixture(autouse=True)
def _no_device_error():
    yield
    if torch.cuda.is_available():
        assert _lib.device_error() == 0


def _ok(status, what):
    assert status == 0, f"{what}: status {status}"


def _d(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return (t if dtype is None else t.to(dtype)).cuda()


def _p(t):
    return None if t is None else t.data_ptr()


class Case:
    """Device inputs of one ensemble shared by both libraries."""

    def __init__(self, rc, cr, angles, starts, grid, geom):
        self.rc, self.cr = rc, cr
        self.ns, self.nc, self.na, self.nt = rc.shape
        self.scan_np = scan_coords(grid)
        self.nv = len(self.scan_np)
        f32 = lambda v: _d(np.asarray(v, np.float32))  # noqa: E731
        self.scan, self.xe, self.ye, self.angles = f32(self.scan_np), f32(geom.x_el), f32(geom.y_el), f32(angles)
        self.starts = f32(np.broadcast_to(np.asarray(starts, np.float32), (self.na,)))
        self.consts = (float(geom.c), float(geom.fs), float(geom.f_demod),
                       -1.0 if geom.fnumber is None else float(geom.fnumber))
        self.drc, self.dcr = _d(rc), _d(cr)
        self.oracle = oracle_inputs(angles, starts, grid, geom)

    def packed(self, handle, half=False):
        elem = 4 if half else 8
        n = self.ns * self.nc * self.na * self.nt
        out = [torch.empty(n * elem, dtype=torch.uint8, device="cuda") for _ in range(2)]
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        for src, dst in zip((self.drc, self.dcr), out):
            if half:
                _ok(handle.rcabeam_pack_ensemble_fp16_device(_p(src), _p(dst), _p(err), self.ns, self.nc, self.na,
                                                             self.nt), "pack fp16")
            else:
                _ok(handle.rcabeam_pack_ensemble_device(_p(src), _p(dst), self.ns, self.nc, self.na, self.nt), "pack")
        return out, err

    def ensemble(self, handle, method=0, half=False, tile=None, signal=True, packed=None):
        """pd (nv,) and signal of one library, called as the reference binding does (voxel tiles)."""
        (prc, pcr), _ = packed if packed is not None else self.packed(handle, half)
        planes = 2 if method == 5 else 1
        nv, nt = self.nv, self.nt
        tile = tile or (16384 if method == 0 else 4096)
        tile = min(tile, nv)
        pd = torch.zeros((nv, 2), dtype=torch.float32, device="cuda")
        sig = torch.zeros((nv * planes, nt), dtype=torch.complex64, device="cuda") if signal else None
        geo = torch.empty(2 * tile * (self.nc + self.na) * 16, dtype=torch.uint8, device="cuda")
        for start in range(0, nv, tile):
            count = min(tile, nv - start)
            scan = self.scan.data_ptr() + 12 * start
            pdp = pd.data_ptr() + 8 * start
            sgp = None if sig is None else sig.data_ptr() + 8 * start * nt * planes
            if half:
                st = handle.rcabeam_opw_fp16_device(_p(prc), _p(pcr), scan, _p(self.xe), _p(self.ye),
                                                    _p(self.angles), _p(self.starts), pdp, sgp, _p(geo), self.ns,
                                                    self.nc, self.na, nt, count, *self.consts)
            else:
                st = handle.rcabeam_ensemble_device(_p(prc), _p(pcr), scan, _p(self.xe), _p(self.ye),
                                                    _p(self.angles), _p(self.starts), pdp, sgp, None, None, _p(geo),
                                                    self.ns, self.nc, self.na, nt, count, *self.consts, method, 2)
            _ok(st, f"ensemble method {method}")
        torch.cuda.synchronize()
        return pd[:, 0].cpu().numpy(), None if sig is None else sig.cpu().numpy()


    def stsw(self, handle, k, tile=4096):
        """St-SW (method 4) XDoppler power and raw weights of one library, in voxel
        tiles with a k^2 nt series workspace per tile (reference python.cpp:553-565)."""
        (prc, pcr), _ = self.packed(handle)
        nv, nt = self.nv, self.nt
        tile = min(tile, nv)
        pd = torch.zeros((nv, 2), dtype=torch.float32, device="cuda")
        weights = torch.zeros(nv, dtype=torch.float32, device="cuda")
        work = torch.empty(tile * k * k * nt, dtype=torch.complex64, device="cuda")
        geo = torch.empty(2 * tile * (self.nc + self.na) * 16, dtype=torch.uint8, device="cuda")
        for start in range(0, nv, tile):
            count = min(tile, nv - start)
            st = handle.rcabeam_ensemble_device(_p(prc), _p(pcr), self.scan.data_ptr() + 12 * start, _p(self.xe),
                                                _p(self.ye), _p(self.angles), _p(self.starts),
                                                pd.data_ptr() + 8 * start, None, weights.data_ptr() + 4 * start,
                                                _p(work), _p(geo), self.ns, self.nc, self.na, nt, count,
                                                *self.consts, 4, k)
            _ok(st, f"St-SW k={k}")
        torch.cuda.synchronize()
        return pd[:, 0].cpu().numpy(), weights.cpu().numpy()


def _random(frames, fnumber, seed=5):
    el = (np.arange(16) - 7.5) * 0.2e-3
    # Offsets keep every |v - e| away from an exact f-number aperture tie: at a
    # tie the reference kernel decides in float32 and its NumPy path (and this
    # library) in float64, which can differ by one whole channel.
    grid = (np.linspace(-1e-3, 1e-3, 5) + 3.71e-5, np.linspace(3e-3, 7e-3, 9) + 1.13e-5,
            np.linspace(-1e-3, 1e-3, 4) + 2.37e-5)
    rc, cr, angles, starts, grid, geom = random_case(seed, 160, 16, 5, frames, grid, fs=20e6, fd=15e6,
                                                     fnumber=fnumber, starts=np.full(5, 3e-6), x_el=el, y_el=el)
    geom = RCAGeometry(el, el, c=1540.0, fs=20e6, f_demod=15e6, fnumber=fnumber)
    return Case(rc, cr, np.deg2rad(np.linspace(-8, 8, 5)), 3e-6, grid, geom)


def test_pack_is_bit_identical(ref):
    rng = np.random.default_rng(2)
    shape = (40, 5, 3, 7)
    rc = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    rc[0, 0, 0, 0] = 1e5  # out of FP16 range: both libraries raise the flag
    case = Case(rc, rc, np.zeros(3), 1e-6, (np.zeros(1), np.array([5e-3]), np.zeros(1)),
                RCAGeometry(np.zeros(5), np.zeros(5)))
    for half in (False, True):
        (a, _), ea = case.packed(ref, half)
        (b, _), eb = case.packed(_lib.lib(), half)
        torch.cuda.synchronize()
        assert torch.equal(a, b)
        assert int(ea.item()) == int(eb.item()) == int(half)


@pytest.mark.parametrize("frames", [8, 33])
@pytest.mark.parametrize("fnumber", [None, 1.0])
@pytest.mark.parametrize("method", [0, 1, 2, 3, 5])
def test_ensemble_methods_match_reference_kernels(ref, method, fnumber, frames):
    case = _random(frames, fnumber)
    pd_ref, sig_ref = case.ensemble(ref, method)
    pd_new, sig_new = case.ensemble(_lib.lib(), method)
    if method == 5:  # separate apertures: IQ only, power untouched (ensemble.cu:278-287)
        assert not pd_ref.any() and not pd_new.any()
    else:
        assert np.abs(pd_ref).max() > 0
        assert rel_l2(pd_new, pd_ref) <= TOL
    if method in (0, 1, 2, 5):
        assert rel_l2(sig_new, sig_ref) <= TOL
    if method == 0:
        o = case.oracle
        iq = das.opw_iq(case.rc, case.cr, o["scan"], o["xe"], o["ye"], o["angles"], o["starts"], o["c"], o["fs"],
                        o["fd"], o["fnumber"])
        err_new, err_ref = rel_l2(sig_new, iq), rel_l2(sig_ref, iq)
        assert err_new <= max(err_ref, 1e-5), (err_new, err_ref)


@pytest.mark.parametrize("frames", [8, 33])
@pytest.mark.parametrize("k", [2, 3, 4])
def test_st_sw_matches_reference_kernels(ref, k, frames):
    """Method 4: XDoppler power, raw weights and the peak-normalized St-SW power of both
    libraries; this build is at least as close to the float64 oracle."""
    case = _random(frames, 1.0)
    pd_ref, w_ref = case.stsw(ref, k)
    pd_new, w_new = case.stsw(_lib.lib(), k)
    assert np.abs(pd_ref).max() > 0 and w_ref.max() > 0
    assert rel_l2(pd_new, pd_ref) <= TOL
    assert rel_l2(w_new, w_ref) <= 1e-3
    power_ref, power_new = pd_ref * w_ref / w_ref.max(), pd_new * w_new / w_new.max()
    assert rel_l2(power_new, power_ref) <= 1e-3  # the reference's St-SW test tolerance
    o = case.oracle
    expected = methods.st_sw_power(case.rc, case.cr, o["scan"], o["xe"], o["ye"], o["angles"], o["starts"], o["c"],
                                   o["fs"], o["fd"], o["fnumber"], k)
    err_new, err_ref = rel_l2(power_new, expected), rel_l2(power_ref, expected)
    assert err_new <= max(err_ref, 1e-4), (err_new, err_ref)


@pytest.mark.parametrize("frames", [8, 64])
def test_fp16_opw_matches_reference_kernel(ref, frames):
    case = _random(frames, None, seed=8)
    pd_ref, sig_ref = case.ensemble(ref, half=True)
    pd_new, sig_new = case.ensemble(_lib.lib(), half=True)
    assert rel_l2(pd_new, pd_ref) <= TOL
    assert rel_l2(sig_new, sig_ref) <= TOL


def test_per_frame_entry_points_match_reference_kernels(ref):
    """Every per-frame entry point of the reference header on one frame of the same channels."""
    case = _random(1, 1.0, seed=11)
    ns, nc, na, nv = case.ns, case.nc, case.na, case.nv
    rc = _d(case.rc[..., 0])
    cr = _d(case.cr[..., 0])
    common = (_p(case.scan), _p(case.xe), _p(case.ye), _p(case.angles), _p(case.starts))
    c = case.consts
    mine = _lib.lib()

    def run(handle, name, n_out, *head, out_dtype=torch.float32, tail=()):
        outs = [torch.zeros(nv, dtype=out_dtype, device="cuda") for _ in range(n_out)]
        _ok(getattr(handle, name)(*head, *[_p(o) for o in outs], ns, nc, na, nv, *tail, *c), name)
        torch.cuda.synchronize()
        return [o.cpu().numpy() for o in outs]

    for name in ("rcabeam_opw_pd_from_channels_device", "rcabeam_xdoppler_pd_from_channels_device",
                 "rcabeam_rc_fmas_pd_from_channels_device", "rcabeam_dmas_ccf_acf_from_channels_device"):
        a = run(ref, name, 1, _p(rc), _p(cr), *common)
        b = run(mine, name, 1, _p(rc), _p(cr), *common)
        assert np.abs(a[0]).max() > 0, name
        assert rel_l2(b[0], a[0]) <= TOL, name
    a = run(ref, "rcabeam_fast_pd_from_channels_device", 3, _p(rc), _p(cr), *common)
    b = run(mine, "rcabeam_fast_pd_from_channels_device", 3, _p(rc), _p(cr), *common)
    for x, y in zip(a, b):
        assert rel_l2(y, x) <= TOL

    # Per-angle volumes of one aperture, then the per-angle IQ reducers on them.
    for config, el in ((0, case.xe), (1, case.ye)):
        src = rc if config == 0 else cr
        vols = []
        for handle in (ref, mine):
            out = torch.zeros((nv, na), dtype=torch.complex64, device="cuda")
            _ok(handle.rcabeam_delay_rca_channels_device(_p(src), _p(case.scan), _p(el), _p(case.angles),
                                                         _p(case.starts), _p(out), ns, nc, na, nv, config, *c),
                "delay_rca_channels")
            chs = torch.zeros((nv, nc), dtype=torch.complex64, device="cuda")
            angs = torch.zeros((nv, na), dtype=torch.complex64, device="cuda")
            act = torch.zeros(nv, dtype=torch.float32, device="cuda")
            _ok(handle.rcabeam_delay_rca_channel_data_device(_p(src), _p(case.scan), _p(el), _p(case.angles),
                                                             _p(case.starts), _p(chs), _p(angs), _p(act), ns, nc, na,
                                                             nv, config, *c), "delay_rca_channel_data")
            torch.cuda.synchronize()
            vols.append((out.cpu().numpy(), chs.cpu().numpy(), angs.cpu().numpy(), act.cpu().numpy()))
        for x, y in zip(*vols):
            assert rel_l2(y, x) <= TOL
        np.testing.assert_array_equal(vols[0][3], vols[1][3])

    rng = np.random.default_rng(4)
    nt = 6
    iq = _d((rng.normal(size=(nv, 2 * na, nt)) + 1j * rng.normal(size=(nv, 2 * na, nt))).astype(np.complex64))
    outs = []
    for handle in (ref, mine):
        o = torch.zeros((nv, nt), dtype=torch.complex64, device="cuda")
        _ok(handle.rcabeam_opw_device(_p(iq), _p(o), nv, 2 * na, nt), "opw")
        xd = torch.zeros(nv, dtype=torch.float32, device="cuda")
        fm = torch.zeros(nv, dtype=torch.float32, device="cuda")
        _ok(handle.rcabeam_xdoppler_pd_device(_p(iq), _p(xd), nv, 2 * na, nt, 0, na, na, na), "xdoppler")
        _ok(handle.rcabeam_rc_fmas_pd_device(_p(iq), _p(fm), nv, 2 * na, nt, 0, na, na, na), "rc_fmas")
        torch.cuda.synchronize()
        outs.append((o.cpu().numpy(), xd.cpu().numpy(), fm.cpu().numpy()))
    for x, y in zip(*outs):
        assert rel_l2(y, x) <= 1e-6


def _time(fn, reps=1):
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def test_full_workload_against_reference_kernels(ref):
    """128+128 el, IQ 512x128x11x200, grid 128x256x128: reference binding loop vs the B200 paths."""
    ns, nc, na, nt = 512, 128, 11, 200
    el = (np.arange(nc) - (nc - 1) / 2) * 0.11e-3
    half = (nc - 1) / 2 * 0.11e-3
    grid = (np.linspace(-half, half, 128), np.linspace(4e-3, 12e-3, 256), np.linspace(-half, half, 128))
    geom = RCAGeometry(el, el, c=1540.0, fs=20e6, f_demod=15e6, fnumber=None)
    angles = np.deg2rad(np.linspace(-10, 10, na))
    gen = torch.Generator(device="cuda").manual_seed(9)
    case = Case.__new__(Case)
    case.ns, case.nc, case.na, case.nt = ns, nc, na, nt
    scan = scan_coords(grid)
    case.nv = len(scan)
    f32 = lambda v: _d(np.asarray(v, np.float32))  # noqa: E731
    case.scan, case.xe, case.ye, case.angles = f32(scan), f32(el), f32(el), f32(angles)
    case.starts = f32(np.full(na, 4e-6))
    case.consts = (1540.0, 20e6, 15e6, -1.0)
    shape = (ns, nc, na, nt)
    case.drc = torch.complex(torch.randn(shape, generator=gen, device="cuda"),
                             torch.randn(shape, generator=gen, device="cuda"))
    case.dcr = torch.complex(torch.randn(shape, generator=gen, device="cuda"),
                             torch.randn(shape, generator=gen, device="cuda"))
    nv = case.nv
    units = nv * 2 * nc * na * nt
    pd = torch.zeros((nv, 2), dtype=torch.float32, device="cuda")
    sig = torch.empty((nv, nt), dtype=torch.complex64, device="cuda")
    rows, outputs = {}, {}

    def reference(half):
        packed = case.packed(ref, half)
        tile = 16384
        geo = torch.empty(2 * tile * (nc + na) * 16, dtype=torch.uint8, device="cuda")
        prc, pcr = packed[0]

        def go():
            for start in range(0, nv, tile):
                args = (_p(prc), _p(pcr), case.scan.data_ptr() + 12 * start, _p(case.xe), _p(case.ye),
                        _p(case.angles), _p(case.starts), pd.data_ptr() + 8 * start, sig.data_ptr() + 8 * start * nt)
                if half:
                    st = ref.rcabeam_opw_fp16_device(*args, _p(geo), ns, nc, na, nt, tile, *case.consts)
                else:
                    st = ref.rcabeam_ensemble_device(*args, None, None, _p(geo), ns, nc, na, nt, tile,
                                                     *case.consts, 0, 2)
                _ok(st, "reference ensemble")
        return go

    def b200(storage):
        hi = [torch.empty(ns * nc * na * nt * (4 if storage != "float32" else 8), dtype=torch.uint8, device="cuda")
              for _ in range(2)]
        lo = [torch.empty_like(hi[0]) for _ in range(2)] if storage == "bf16x2" else None
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        mine = _lib.lib()
        for i, src in enumerate((case.drc, case.dcr)):
            if storage == "bf16x2":
                _ok(mine.rcabeam_pack_ensemble_split_device(_p(src), _p(hi[i]), _p(lo[i]), _p(err), ns, nc, na, nt),
                    "split")
            elif storage == "float16":
                _ok(mine.rcabeam_pack_ensemble_fp16_device(_p(src), _p(hi[i]), _p(err), ns, nc, na, nt), "fp16")
            else:
                _ok(mine.rcabeam_pack_ensemble_device(_p(src), _p(hi[i]), ns, nc, na, nt), "pack")
        geo = torch.empty(_cuda_impl.workspace_bytes(nv, nc, na), dtype=torch.uint8, device="cuda")
        common = (_p(case.scan), _p(case.xe), _p(case.ye), _p(case.angles), _p(case.starts), _p(pd), _p(sig))

        def go():
            if storage == "bf16x2":
                st = mine.rcabeam_opw_tc_device(_p(hi[0]), _p(lo[0]), _p(hi[1]), _p(lo[1]), *common, _p(geo), ns, nc,
                                                na, nt, nv, *case.consts, 1)
            elif storage == "float16":
                st = mine.rcabeam_opw_fp16_device(_p(hi[0]), _p(hi[1]), *common, _p(geo), ns, nc, na, nt, nv,
                                                  *case.consts)
            else:
                st = mine.rcabeam_ensemble_device(_p(hi[0]), _p(hi[1]), *common, None, None, _p(geo), ns, nc, na, nt,
                                                  nv, *case.consts, 0, 2)
            _ok(st, f"b200 {storage}")
        return go

    for name, make in (("reference float32", lambda: reference(False)), ("reference float16", lambda: reference(True)),
                       ("b200 float32 (staged SIMT)", lambda: b200("float32")),
                       ("b200 float16 (tcgen05)", lambda: b200("float16")),
                       ("b200 bf16x2 (tcgen05, 3 products)", lambda: b200("bf16x2"))):
        go = make()
        ms = _time(go)
        rows[name] = ms
        outputs[name] = pd[:, 0].clone()
        torch.cuda.empty_cache()
    print("\nOPW DAS, full workload (IQ + power written), one ensemble:")
    for name, ms in rows.items():
        print(f"  {name:36s} {ms:9.1f} ms  {units / ms / 1e6:8.1f} Gsamples/s")
    base = outputs["reference float32"]
    for name in ("b200 float32 (staged SIMT)", "b200 bf16x2 (tcgen05, 3 products)"):
        err = float(torch.linalg.vector_norm(outputs[name] - base) / torch.linalg.vector_norm(base))
        print(f"  power rel. L2 {name} vs reference float32: {err:.2e}")
        assert err <= TOL
    err = float(torch.linalg.vector_norm(outputs["b200 float16 (tcgen05)"] - outputs["reference float16"])
                / torch.linalg.vector_norm(outputs["reference float16"]))
    print(f"  power rel. L2 b200 float16 vs reference float16: {err:.2e}")
    assert err <= TOL
    assert rows["b200 bf16x2 (tcgen05, 3 products)"] < rows["reference float32"]
    assert rows["b200 float16 (tcgen05)"] < rows["reference float16"]


def _full_block_case():
    """The full workload's channels (IQ 512x128x11x200) on its central 32 x 64 x 32 voxel block."""
    ns, nc, na, nt = 512, 128, 11, 200
    el = (np.arange(nc) - (nc - 1) / 2) * 0.11e-3
    half = (nc - 1) / 2 * 0.11e-3
    axes = (np.linspace(-half, half, 128), np.linspace(4e-3, 12e-3, 256), np.linspace(-half, half, 128))
    grid = tuple(a[(len(a) - n) // 2:(len(a) - n) // 2 + n] for a, n in zip(axes, (32, 64, 32)))
    angles = np.deg2rad(np.linspace(-10, 10, na))
    gen = torch.Generator(device="cuda").manual_seed(9)
    case = Case.__new__(Case)
    case.ns, case.nc, case.na, case.nt = ns, nc, na, nt
    scan = scan_coords(grid)
    case.nv = len(scan)
    f32 = lambda v: _d(np.asarray(v, np.float32))  # noqa: E731
    case.scan, case.xe, case.ye, case.angles = f32(scan), f32(el), f32(el), f32(angles)
    case.starts = f32(np.full(na, 4e-6))
    case.consts = (1540.0, 20e6, 15e6, -1.0)
    shape = (ns, nc, na, nt)
    case.drc = torch.complex(torch.randn(shape, generator=gen, device="cuda"),
                             torch.randn(shape, generator=gen, device="cuda"))
    case.dcr = torch.complex(torch.randn(shape, generator=gen, device="cuda"),
                             torch.randn(shape, generator=gen, device="cuda"))
    return case


def test_st_sw_block_against_reference_kernels(ref):
    """St-SW k = 2 on the central block of the full workload: both libraries through the C ABI in
    4096-voxel tiles with a k^2 nt series workspace (the reference binding's tiling,
    python.cpp:553-565); power agreement and both times (printed)."""
    case, k = _full_block_case(), 2
    shape = (case.ns, case.nc, case.na, case.nt)
    units = case.nv * 2 * case.nc * case.na * case.nt
    results = {}
    for name, handle in (("reference", ref), ("b200", _lib.lib())):
        case.stsw(handle, k)  # warm-up (includes packing)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        pd, w = case.stsw(handle, k)
        b.record()
        torch.cuda.synchronize()
        results[name] = (a.elapsed_time(b), pd * w / w.max())
    err = rel_l2(results["b200"][1], results["reference"][1])
    print(f"\nSt-SW k={k}, {case.nv} voxels, IQ {shape}, packing + series + finish, 4096-voxel tiles:")
    for name, (ms, _) in results.items():
        print(f"  {name:10s} {ms:9.1f} ms  {units / ms / 1e6:8.1f} Gsamples/s")
    print(f"  St-SW power rel. L2 b200 vs reference: {err:.2e}")
    assert err <= 1e-3


@pytest.mark.parametrize("method,label", [(2, "RC-FMAS"), (3, "DMAS-CCF-ACF")])
def test_nonlinear_block_against_reference_kernels(ref, method, label):
    """RC-FMAS (method 2) and DMAS-CCF-ACF (method 3) on the central block of the full workload,
    signal and power written, both libraries in the reference binding's 4096-voxel tiles:
    agreement and both times (printed)."""
    case = _full_block_case()
    units = case.nv * 2 * case.nc * case.na * case.nt
    results = {}
    for name, handle in (("reference", ref), ("b200", _lib.lib())):
        packed = case.packed(handle)
        case.ensemble(handle, method=method, packed=packed)  # warm-up
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        pd, sig = case.ensemble(handle, method=method, packed=packed)
        b.record()
        torch.cuda.synchronize()
        results[name] = (a.elapsed_time(b), pd, sig)
    print(f"\n{label}, {case.nv} voxels, IQ {(case.ns, case.nc, case.na, case.nt)}, signal + power, "
          "4096-voxel tiles:")
    for name, (ms, *_) in results.items():
        print(f"  {name:10s} {ms:9.1f} ms  {units / ms / 1e6:8.1f} Gsamples/s")
    assert rel_l2(results["b200"][1], results["reference"][1]) <= TOL
    assert rel_l2(results["b200"][2], results["reference"][2]) <= TOL
