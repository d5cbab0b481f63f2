"""GPU test of nwprt_sh_project_static, the SH projection that allocates no device memory.

Callers such as a real-time frame loop (cudaMalloc/cudaFree can synchronise the device and
stall a frame) or a host that reserves all device memory up front cannot hand the
projection a workspace; this entry point keeps its partial sums in a fixed static device
array instead.  Its result must match nwprt_sh_project (caller workspace) within the
tolerance the SH tests use, call after call, although every call reuses the same array.
"""
import ctypes as C

import numpy as np
import pytest

from neural_wavelet_prt_demo_b200 import synth

pytestmark = pytest.mark.gpu


def _project_with_workspace(lib, faces, S):
    import torch
    nbytes = lib.nwprt_sh_project_workspace_size(S)
    ws = torch.empty(nbytes // 4, dtype=torch.float32, device=faces.device)
    L = torch.empty((81, 3), dtype=torch.float32, device=faces.device)
    s = lib.nwprt_sh_project(C.c_void_p(faces.data_ptr()), S, C.c_void_p(L.data_ptr()),
                             C.c_void_p(ws.data_ptr()), nbytes, None)
    return s, L


def _project_static(lib, faces, S):
    import torch
    L = torch.full((81, 3), float("nan"), dtype=torch.float32, device=faces.device)
    s = lib.nwprt_sh_project_static(C.c_void_p(faces.data_ptr()), S, C.c_void_p(L.data_ptr()), None)
    return s, L


def test_static_projection_matches_workspace_projection_on_consecutive_calls(cuda):
    import torch
    from neural_wavelet_prt_demo_b200 import _lib
    lib = _lib.lib()
    # two calls in a row on different cubemaps: the second must not see the first's partial sums
    for S, seed in ((128, 11), (64, 12), (128, 13)):
        faces = torch.from_numpy(synth.make_env_faces(S, seed=seed)).to(cuda)
        s_static, L_static = _project_static(lib, faces, S)
        assert s_static == _lib.OK, lib.nwprt_last_error(None)
        s_ref, L_ref = _project_with_workspace(lib, faces, S)
        assert s_ref == _lib.OK
        torch.cuda.synchronize()
        got, ref = L_static.cpu().numpy(), L_ref.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert np.allclose(got, ref, rtol=1e-5, atol=1e-7 * float(np.abs(ref).max()))


def test_static_projection_allocates_nothing(cuda):
    """After a first call (which loads the module and looks up the array's address), further
    calls leave the device's free memory unchanged: the partial sums never need an
    allocation, which is what callers that cannot allocate rely on.  S = 100 also checks a
    face size that is not a power of two, and a call from a new host thread checks that no
    per-thread set-up is needed."""
    import threading
    import torch
    from neural_wavelet_prt_demo_b200 import _lib
    lib = _lib.lib()
    S = 100
    faces = torch.from_numpy(synth.make_env_faces(S, seed=21)).to(cuda)
    s_ref, L_ref = _project_with_workspace(lib, faces, S)
    assert s_ref == _lib.OK
    L = torch.full((81, 3), float("nan"), dtype=torch.float32, device=cuda)
    args = (C.c_void_p(faces.data_ptr()), S, C.c_void_p(L.data_ptr()), None)
    assert lib.nwprt_sh_project_static(*args) == _lib.OK
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        assert lib.nwprt_sh_project_static(*args) == _lib.OK
    statuses = []
    t = threading.Thread(target=lambda: statuses.append(lib.nwprt_sh_project_static(*args)))
    t.start()
    t.join()
    assert statuses == [_lib.OK]
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before, (free_before, free_after)
    got, ref = L.cpu().numpy(), L_ref.cpu().numpy()
    assert np.allclose(got, ref, rtol=1e-5, atol=1e-7 * float(np.abs(ref).max()))


def test_static_projection_rejects_faces_beyond_its_scratch(cuda):
    import torch
    from neural_wavelet_prt_demo_b200 import _lib
    lib = _lib.lib()
    faces = torch.zeros((6, 256, 256, 3), dtype=torch.float32, device=cuda)
    L = torch.zeros((81, 3), dtype=torch.float32, device=cuda)
    s = lib.nwprt_sh_project_static(C.c_void_p(faces.data_ptr()), 256, C.c_void_p(L.data_ptr()), None)
    assert s == _lib.INVALID_ARG
    assert b"128" in lib.nwprt_last_error(None)
