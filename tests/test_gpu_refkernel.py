"""The reference's own GPU Legendre kernel (all_transpose_legendre_transforms,
wavemoth/cuda/legendre_transform.cu.in:643-679, built from its template by
oracle/Makefile) against this library's map2alm Legendre phase on the same
q, on the dense-recurrence plan (the reference kernel's scheme).

Correctness (nside 128, lmax 256, 1 map): this library's a = Lambda^T q
against the exact dense product of the oracle (1e-11 relative L2); the
reference kernel's output against the same (recorded, and required within
1e-8: its reduction is written warp-synchronously for pre-Volta GPUs).

Timing (WAVEMOTH_REF_KERNEL_TIMING=1; nside 1024, lmax 2048, the reference
kernel's one map): both kernels' device times, written to
$WAVEMOTH_PROFILE_OUT/refkernel_nside1024.json when that is set.
"""
import json
import os

import numpy as np
import pytest

from oracle import sht as osht

from .plans import plan_file, rel

pytestmark = pytest.mark.gpu


def _setup(nside, lmax, torch):
    from oracle import refgpu
    ni = 2 * nside
    if not refgpu.available(ni):
        pytest.skip("reference GPU kernel not built for %d rings" % ni)
    res, nnz = refgpu.resource(nside, lmax)
    rng = np.random.default_rng(1)
    q = rng.standard_normal((lmax + 1, 2, 2, ni))
    d_res = torch.from_numpy(res).cuda()
    d_q = torch.from_numpy(q).cuda()
    # this library's q: [ring][m][parity][vector]
    d_q_ours = d_q.permute(3, 0, 1, 2).contiguous()
    return refgpu, ni, nnz, q, d_res, d_q, d_q_ours


def _ours(T, d_q_ours, torch):
    from wavemoth_b200 import _native
    out = torch.empty((T.nalm, T.nmaps), dtype=torch.complex128, device="cuda")
    rc = _native.lib().wavemoth_legendre_map2alm_device(T.plan_handle, d_q_ours.data_ptr(), out.data_ptr(),
                                                         torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    return out


def test_reference_kernel_matches():
    torch = pytest.importorskip("torch")
    from wavemoth_b200.sht import Transform
    nside, lmax = 128, 256
    refgpu, ni, nnz, q, d_res, d_q, d_q_ours = _setup(nside, lmax, torch)
    nalm = (lmax + 1) * (lmax + 2) // 2
    a_ref = torch.zeros((nalm, 2), dtype=torch.float64, device="cuda")
    refgpu.all_transpose(ni, lmax, d_res.data_ptr(), d_q.data_ptr(), a_ref.data_ptr())
    T = Transform(None, nside, lmax, 1, dense=True)
    a = _ours(T, d_q_ours, torch)
    torch.cuda.synchronize()
    T.close()
    # exact: a_lm = sum_i lambda_lm(theta_i) q[m, parity(l - m), :, i]
    work = np.ascontiguousarray(q.transpose(0, 1, 3, 2)).view(np.complex128)[..., 0][..., None]
    want = osht.legendre_phase_adjoint_dense(nside, work, lmax)
    got = a.cpu().numpy()
    assert rel(got, want) < 1e-11
    got_ref = a_ref.cpu().numpy().view(np.complex128)
    assert rel(got_ref, want) < 1e-8


@pytest.mark.skipif(os.environ.get("WAVEMOTH_REF_KERNEL_TIMING") != "1", reason="timing run on request")
def test_reference_kernel_timing_nside1024():
    torch = pytest.importorskip("torch")
    from wavemoth_b200.sht import Transform
    nside, lmax = 1024, 2048
    refgpu, ni, nnz, q, d_res, d_q, d_q_ours = _setup(nside, lmax, torch)
    nalm = (lmax + 1) * (lmax + 2) // 2
    a_ref = torch.zeros((nalm, 2), dtype=torch.float64, device="cuda")

    def timed(fn, n=5):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    ms_ref = timed(lambda: refgpu.all_transpose(ni, lmax, d_res.data_ptr(), d_q.data_ptr(), a_ref.data_ptr(),
                                                torch.cuda.current_stream().cuda_stream))
    out = {"nside": nside, "lmax": lmax, "reference_kernel_1map_ms": ms_ref,
           "reference_flops_1map": nnz * (5 + 2 * 2), "flop_convention": "nnz (5 + 2 nvecs), cuda/sht.py:155-159"}
    D = Transform(None, nside, lmax, 1, dense=True)
    out["ours_dense_1map_ms"] = timed(lambda: _ours(D, d_q_ours, torch))
    a = _ours(D, d_q_ours, torch)
    torch.cuda.synchronize()
    out["rel_l2_ours_vs_reference_kernel"] = rel(a.cpu().numpy(), a_ref.cpu().numpy().view(np.complex128))
    D.close()
    path = plan_file(nside, lmax, 64, 1e-10, 20.0, workers=min(len(os.sched_getaffinity(0)), 32))
    for nmaps in (1, 32):
        qq = d_q_ours.repeat_interleave(nmaps, dim=3) if nmaps > 1 else d_q_ours
        qq = qq.reshape(ni, lmax + 1, 2, 2 * nmaps).contiguous()
        for prec in ("double", "split"):
            B = Transform(path, nside, lmax, nmaps, precision=prec)
            out["ours_butterfly_%s_%dmaps_ms" % (prec, nmaps)] = timed(lambda: _ours(B, qq, torch))
            B.close()
        if nmaps == 32:
            D = Transform(None, nside, lmax, nmaps, dense=True)
            out["ours_dense_32maps_ms"] = timed(lambda: _ours(D, qq, torch))
            D.close()
    dest = os.environ.get("WAVEMOTH_PROFILE_OUT")
    if dest:
        os.makedirs(dest, exist_ok=True)
        with open(os.path.join(dest, "refkernel_nside1024.json"), "w") as f:
            json.dump(out, f, indent=1)
    print(json.dumps(out))
