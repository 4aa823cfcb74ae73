"""md_lj_forces_static: the Lennard-Jones entry point for callers that cannot
allocate device memory (a framework that owns all device memory through its own
pool, latency-critical loops that cannot afford a device-wide synchronisation from
cudaMalloc).  The caller passes device buffers; the library's only working memory
is a fixed array in its device image.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.  It passes alone in a fresh
process and after the other tests (its first call resolves the array's address).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def approx_eq(a, b, eps=1e-12):
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    return np.all(np.abs(a - b) < eps * (1.0 + np.maximum(np.abs(a), np.abs(b))))


def device_buffers(torch, pos):
    """The caller's device memory: positions and NaN-filled outputs (torch-owned)."""
    n = pos.shape[0]
    dev = torch.device("cuda", 0)
    x, y, z = (torch.tensor(np.ascontiguousarray(pos[:, k]), dtype=torch.float64, device=dev)
               for k in range(3))
    f = [torch.full((n,), float("nan"), dtype=torch.float64, device=dev) for _ in range(3)]
    ev = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
    return (x, y, z), f, ev


def launch(md, bufs, n, box, trunc, stream=None):
    (x, y, z), f, ev = bufs
    b = np.ascontiguousarray(box, dtype=np.float64)
    ptr = (lambda t: t.data_ptr()) if n > 0 else (lambda t: None)
    return md.lib().md_lj_forces_static(
        ptr(x), ptr(y), ptr(z), n, b.ctypes.data_as(C.POINTER(C.c_double)), 1.0, 1.0, 2.5, trunc,
        ptr(f[0]), ptr(f[1]), ptr(f[2]), ev.data_ptr(), stream)


def static_call(md, torch, pos, box, trunc, stream=None):
    """One call of the entry point on torch-owned device buffers (the caller's memory),
    on the legacy default stream or on the given torch stream."""
    n = pos.shape[0]
    bufs = device_buffers(torch, pos)
    f, ev = bufs[1], bufs[2]
    torch.cuda.synchronize()
    md._check(launch(md, bufs, n, box, trunc, stream.cuda_stream if stream is not None else None))
    torch.cuda.synchronize()
    forces = np.stack([t.cpu().numpy() for t in f], 1)
    e, w = ev.cpu().numpy()
    return forces, e, w


def test_static_scratch_entry_point_matches_md_lj_forces(md):
    torch = pytest.importorskip("torch")
    st = md.fcc_lattice(6, 0.8442, 0.722, 3)  # N = 864
    rng = np.random.default_rng(5)
    box = st["box"]
    # two calls in a row, on different states and truncations, each checked
    # against the existing entry point (md_lj_forces through an md_system)
    for call, trunc in enumerate((md.Truncation.Truncated, md.Truncation.LinearForceShift)):
        pos = st["pos"] + rng.normal(scale=0.08 * (call + 1), size=st["pos"].shape)
        pos -= box * np.floor(pos / box + 0.5)
        sys_ = md.System.from_arrays(pos, box)
        e_ref, w_ref = md.LennardJones(1.0, 1.0, 2.5, trunc).compute_forces(sys_)
        f_ref = sys_.forces
        f, e, w = static_call(md, torch, pos, box, trunc)
        assert approx_eq(f, f_ref), call
        assert approx_eq(e, e_ref) and approx_eq(w, w_ref), (call, e, e_ref, w, w_ref)


def test_static_scratch_side_stream_and_unwrapped_positions(md):
    """On a caller's stream, positions shifted by whole boxes (not wrapped): the same
    forces, energy and virial as md_lj_forces on the wrapped state, twice in a row."""
    torch = pytest.importorskip("torch")
    st = md.fcc_lattice(5, 0.8442, 0.722, 9)  # N = 500
    box = st["box"]
    rng = np.random.default_rng(9)
    pos = st["pos"] + rng.normal(scale=0.05, size=st["pos"].shape)
    pos -= box * np.floor(pos / box + 0.5)
    sys_ = md.System.from_arrays(pos, box)
    e_ref, w_ref = md.LennardJones(1.0, 1.0, 2.5).compute_forces(sys_)
    f_ref = sys_.forces
    shifted = pos + box * rng.integers(-3, 4, size=pos.shape)
    stream = torch.cuda.Stream()
    for _ in range(2):
        f, e, w = static_call(md, torch, shifted, box, md.Truncation.Truncated, stream)
        assert approx_eq(f, f_ref) and approx_eq(e, e_ref) and approx_eq(w, w_ref)


def test_static_scratch_empty_system_and_no_device_memory_taken(md):
    """n = 0 writes zero energy and virial; a call after the first takes no device
    memory (the free device memory is unchanged across it)."""
    torch = pytest.importorskip("torch")
    box = np.array([8.0, 8.0, 8.0])
    bufs = device_buffers(torch, np.zeros((0, 3)))
    md._check(launch(md, bufs, 0, box, 0))
    torch.cuda.synchronize()
    assert np.array_equal(bufs[2].cpu().numpy(), [0.0, 0.0])
    st = md.fcc_lattice(4, 0.8442, 0.722, 2)
    bufs = device_buffers(torch, st["pos"])
    md._check(launch(md, bufs, st["pos"].shape[0], st["box"], 0))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    md._check(launch(md, bufs, st["pos"].shape[0], st["box"], 0))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_static_scratch_rejects_oversized_systems(md):
    box = np.array([10.0, 10.0, 10.0])
    rc = md.lib().md_lj_forces_static(None, None, None, 262145, box.ctypes.data_as(
        C.POINTER(C.c_double)), 1.0, 1.0, 2.5, 0, None, None, None, None, None)
    assert rc == md.MD_ERR_INVALID_ARGUMENT
    msg = md.lib().md_last_error().decode()
    assert "262144" in msg or "262,144" in msg or "exceeds" in msg
    rc = md.lib().md_lj_forces_static(None, None, None, -1, box.ctypes.data_as(
        C.POINTER(C.c_double)), 1.0, 1.0, 2.5, 0, None, None, None, None, None)
    assert rc == md.MD_ERR_INVALID_ARGUMENT
    assert "non-negative" in md.lib().md_last_error().decode()
