"""CPU checks of the drop-in boundary: the libraries load, export every entry
point include/*.h declares (and nothing the reference lacks is missing), and
the host-only loaders behave like the reference's.  No device computation."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg

ROOT = Path(__file__).resolve().parent.parent


def _declared(header: Path):
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b(pf\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_kernel_library_exports_header():
    lib = pkg.kernels()
    names = _declared(ROOT / "include" / "pfc_abi.h")
    assert len(names) >= 40
    for name in names:
        assert hasattr(lib, name), name


def test_drop_in_symbols_present():
    lib = pkg.kernels()
    for name in pkg.PF_ABI_SYMBOLS:
        assert hasattr(lib, name), name
    assert len(pkg.PF_ABI_SYMBOLS) == 18


def test_core_library_exports_header():
    lib = pkg.core()
    names = _declared(ROOT / "include" / "pf_core.h")
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name


def test_struct_layouts():
    # repr(C) CObservation of crates/pf_core/src/cuda.rs:18-27
    assert C.sizeof(pkg.CObservation) == 24
    assert pkg.CObservation.dx.offset == 8
    assert pkg.CObservation.range.offset == 20


def test_version_and_null_handles():
    lib = pkg.kernels()
    assert lib.pfc_version() >= 100
    assert lib.pfc_destroy(None) == 0
    assert lib.pfgl_destroy(None) == 0
    assert lib.pfgl_free_cells(None) == -1
    assert lib.pfc_init(None, 10, 1) == -1
    assert lib.pfc_est_sums(None, None) == -1


def test_quat_mean_host_matches_numpy():
    lib = pkg.core()
    rng = np.random.default_rng(1)
    q = rng.normal(size=(200, 4)) * 0.1 + np.array([0.2, 0.9, 0.1, -0.3])
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    m = (q[:, :, None] * q[:, None, :]).mean(0)
    m10 = np.array([m[r, c] for r in range(4) for c in range(r, 4)])
    out = np.zeros(4)
    lib.pfcore_quat_mean(pkg.dptr(m10), pkg.dptr(out))
    vals, vecs = np.linalg.eigh(m)
    ref = vecs[:, np.argmax(vals)]
    ref = ref if ref[0] >= 0 else -ref
    assert np.allclose(out, ref, atol=1e-12)


def _pgm(w, h, px: np.ndarray, comment=True):
    hdr = b"P5\n" + (b"# made by test\n" if comment else b"") + f"{w} {h}\n255\n".encode()
    return hdr + px.astype(np.uint8).tobytes()


def test_pgm_yaml_loader_flips_rows_and_thresholds():
    # OccGrid::from_pgm_yaml, crates/pf_core/src/global_loc.rs:30-130
    lib = pkg.core()
    w, h = 5, 3
    px = np.full((h, w), 254, np.uint8)
    px[0, 1] = 0      # top row in the image -> last row of the grid
    px[2, 3] = 100    # (255-100)/255 = 0.61 < 0.65: free
    px[1, 4] = 50     # 0.80 > 0.65: occupied
    data = _pgm(w, h, px)
    yaml = b"image: m.pgm\nresolution: 0.1 # m\norigin: [-1.5, 2.0, 0.0]\noccupied_thresh: 0.65\n"
    W, H = C.c_int(), C.c_int()
    res, ox, oy = C.c_double(), C.c_double(), C.c_double()
    assert lib.pfcore_grid_from_pgm_yaml(data, len(data), yaml, C.byref(W), C.byref(H),
                                         C.byref(res), C.byref(ox), C.byref(oy), None) == 0
    assert (W.value, H.value) == (w, h)
    assert res.value == 0.1 and ox.value == -1.5 and oy.value == 2.0
    cells = np.zeros(w * h, np.uint8)
    assert lib.pfcore_grid_from_pgm_yaml(data, len(data), yaml, C.byref(W), C.byref(H),
                                         C.byref(res), C.byref(ox), C.byref(oy),
                                         pkg.u8ptr(cells)) == 0
    g = cells.reshape(h, w)
    assert g[2, 1] == 1 and g[0, 3] == 0 and g[1, 4] == 1
    assert g.sum() == 2


def test_pgm_yaml_loader_rejects_bad_input():
    lib = pkg.core()
    W, H = C.c_int(), C.c_int()
    res, ox, oy = C.c_double(), C.c_double(), C.c_double()
    args = (C.byref(W), C.byref(H), C.byref(res), C.byref(ox), C.byref(oy), None)
    good_yaml = b"resolution: 0.05\norigin: [0, 0, 0]\n"
    bad = b"P2\n2 2\n255\n0000"
    assert lib.pfcore_grid_from_pgm_yaml(bad, len(bad), good_yaml, *args) == -1
    short = b"P5\n4 4\n255\n" + b"\x00" * 5
    assert lib.pfcore_grid_from_pgm_yaml(short, len(short), good_yaml, *args) == -1
    ok = _pgm(2, 2, np.zeros((2, 2)))
    assert lib.pfcore_grid_from_pgm_yaml(ok, len(ok), b"origin: [0,0,0]\n", *args) == -1
    assert lib.pfcore_grid_from_pgm_yaml(ok, len(ok), b"resolution: 0.05\n", *args) == -1
