"""tcgen05 BF16 GEMMs against an fp32 product of the same bf16 inputs:
sphg_gemm_bf16_tn (C = A B^T, accumulate, split-K, every N tile width) and
the weight-stationary persistent sphg_gemm_bf16_ws with each fused epilogue,
from one tile to many tiles per CTA."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K,acc,split", [(128, 128, 64, 0, 1), (256, 128, 192, 0, 1), (384, 64, 256, 1, 1),
                                             (128, 16, 128, 0, 1), (256, 32, 64, 0, 1), (128, 384, 320, 0, 1),
                                             (512, 128, 1024, 1, 4), (128, 48, 64, 0, 1)])
def test_gemm_matches_fp32_reference(cuda_ok, lib, M, N, K, acc, split):
    import torch
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C0 = torch.randn(M, N, device="cuda", generator=g)
    C = C0.clone() if (acc or split > 1) else torch.zeros(M, N, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.sphg_gemm_bf16_tn(A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K, acc, split, err.data_ptr(),
                               torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rc == 0 and int(err.item()) == 0
    ref = A.float() @ B.float().T
    if acc or split > 1:
        ref = ref + C0
    scale = float(ref.abs().max())
    assert float((C - ref).abs().max()) <= 1e-4 * scale * (K / 64) ** 0.5, float((C - ref).abs().max()) / scale


def test_gemm_rejects_bad_shapes(lib):
    import ctypes
    one = ctypes.c_void_p(16)
    assert lib.sphg_gemm_bf16_tn(one, one, one, 100, 128, 64, 0, 1, one, None) != 0   # M % 128
    assert lib.sphg_gemm_bf16_tn(one, one, one, 128, 24, 64, 0, 1, one, None) != 0    # N % 16
    assert lib.sphg_gemm_bf16_tn(one, one, one, 128, 128, 32, 0, 1, one, None) != 0   # K % 64


WS_SHAPES = [(128, 64), (128, 128), (256, 128), (128, 256)]


def _ws(lib, A, B, M, N, K, epi):
    import torch
    from sources_b200 import learn
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.sphg_gemm_bf16_ws(A.data_ptr(), B.data_ptr(), M, N, K, ctypes_addr(epi), err.data_ptr(),
                               torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rc == 0 and int(err.item()) == 0


def ctypes_addr(s):
    import ctypes
    return ctypes.addressof(s)


@pytest.mark.parametrize("N,K", WS_SHAPES)
@pytest.mark.parametrize("M", [128, 640, 128 * 701])
def test_ws_gemm_epilogues(cuda_ok, lib, M, N, K):
    import torch
    from sources_b200 import learn
    g = torch.Generator(device="cuda").manual_seed(M + 3 * N + 7 * K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = (torch.randn(N, K, device="cuda", generator=g) / K ** 0.5).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    prod = A.float() @ B.float().T
    tol = 1e-4 * float(prod.abs().max()) * (K / 64) ** 0.5 + 1e-5
    E = learn.GemmEpi()
    # STORE
    z = torch.full((M, N), float("nan"), device="cuda")
    E.mode, E.z = learn.EPI_STORE, z.data_ptr()
    _ws(lib, A, B, M, N, K, E)
    assert float((z - prod).abs().max()) <= tol
    # ACC
    z0 = torch.randn(M, N, device="cuda", generator=g)
    z = z0.clone()
    E.mode = learn.EPI_ACC
    E.z = z.data_ptr()
    _ws(lib, A, B, M, N, K, E)
    assert float((z - (z0 + prod)).abs().max()) <= tol
    # BIAS_ACT with and without relu, z kept or not
    for relu, keep in ((1, True), (0, False)):
        z = torch.zeros(M, N, device="cuda")
        h = torch.zeros(M, N, device="cuda", dtype=torch.bfloat16)
        E = learn.GemmEpi(mode=learn.EPI_BIAS_ACT, relu=relu, bias=bias.data_ptr(), z=z.data_ptr() if keep else None,
                          h=h.data_ptr())
        _ws(lib, A, B, M, N, K, E)
        ref = prod + bias
        if keep:
            assert float((z - ref).abs().max()) <= tol
        else:
            assert not z.any()
        act = ref.clamp_min(0) if relu else ref
        assert float((h.float() - act).abs().max()) <= 1e-2 * float(act.abs().max()) + tol
    # EDGE: rows beyond nedge get the bias only
    nodes = 300
    P = torch.randn(nodes, 2 * N, device="cuda", generator=g)
    nedge = M - 37 if M > 128 else M
    src = torch.randint(0, nodes, (M,), device="cuda", generator=g, dtype=torch.int32)
    dst = torch.randint(0, nodes, (M,), device="cuda", generator=g, dtype=torch.int32)
    z = torch.zeros(M, N, device="cuda")
    h = torch.zeros(M, N, device="cuda", dtype=torch.bfloat16)
    E = learn.GemmEpi(mode=learn.EPI_EDGE, relu=1, bias=bias.data_ptr(), z=z.data_ptr(), h=h.data_ptr(),
                      P=P.data_ptr(), src=src.data_ptr(), dst=dst.data_ptr(), nedge=nedge)
    _ws(lib, A, B, M, N, K, E)
    ref = prod + bias
    ref[:nedge] += P[src[:nedge].long(), :N] + P[dst[:nedge].long(), N:]
    assert float((z - ref).abs().max()) <= tol
    assert float((h.float() - ref.clamp_min(0)).abs().max()) <= 1e-2 * float(ref.abs().max()) + tol
    # RESID
    z0 = torch.randn(M, N, device="cuda", generator=g)
    z = z0.clone()
    h = torch.zeros(M, N, device="cuda", dtype=torch.bfloat16)
    E = learn.GemmEpi(mode=learn.EPI_RESID, bias=bias.data_ptr(), z=z.data_ptr(), h=h.data_ptr())
    _ws(lib, A, B, M, N, K, E)
    ref = z0 + prod + bias
    assert float((z - ref).abs().max()) <= tol
    assert float((h.float() - ref).abs().max()) <= 1e-2 * float(ref.abs().max()) + tol


def test_ws_gemm_rejects_bad_arguments(lib):
    from sources_b200 import learn
    import ctypes
    one = ctypes.c_void_p(256)
    E = learn.GemmEpi(mode=learn.EPI_STORE, z=256)
    a = ctypes.addressof(E)
    assert lib.sphg_gemm_bf16_ws(one, one, 100, 128, 128, a, one, None) != 0      # M % 128
    assert lib.sphg_gemm_bf16_ws(one, one, 128, 64, 128, a, one, None) != 0      # unsupported (N, K)
    E.z = None
    assert lib.sphg_gemm_bf16_ws(one, one, 128, 128, 128, a, one, None) != 0     # STORE without z
    E.mode = 9
    assert lib.sphg_gemm_bf16_ws(one, one, 128, 128, 128, a, one, None) != 0     # unknown epilogue


def test_bounded_wait_runs_out_and_frees_tmem(cuda_ok, lib):
    """A device wait that gives up: sphg_gemm_wait_probe launches the GEMM
    kernel so that its first mbarrier wait has nothing to wait for and runs
    out after 2,000 polls, before any MMA or copy is in flight.  The call
    returns SPHG_ERR_TIMEOUT with the error flag set; the kernel freed its
    TMEM, so ordinary GEMMs on the same SMs afterwards allocate TMEM again and
    give the right product (twice, around a second probe)."""
    import torch
    from sources_b200.abi import SPHG_ERR_TIMEOUT
    M, N, K = 128 * 296, 128, 128      # two CTAs per SM on every SM
    g = torch.Generator(device="cuda").manual_seed(7)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    ref = A.float() @ B.float().T
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        rc = lib.sphg_gemm_wait_probe(A.data_ptr(), B.data_ptr(), M, N, K, 2000, err.data_ptr(), stream)
        assert rc == SPHG_ERR_TIMEOUT and int(err.item()) == 1
        err.zero_()
        C = torch.zeros(M, N, device="cuda")
        assert lib.sphg_gemm_bf16_tn(A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K, 0, 1, err.data_ptr(),
                                     stream) == 0
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        assert float((C - ref).abs().max()) <= 1e-4 * float(ref.abs().max()) * (K / 64) ** 0.5


@pytest.mark.parametrize("M,inplace", [(128, False), (128 * 5, True), (128 * 1201, True), (128 * 1201, False)])
def test_fused_edge_layer_equals_two_gemms(cuda_ok, lib, M, inplace):
    """sphg_gnn_edge_layer (edge GEMM, ReLU and residual GEMM in one kernel,
    the hidden rows kept in shared memory) gives the same bits as the two
    weight-stationary GEMMs with the EDGE and RESID epilogues, padding rows
    (beyond nedge) included; E may be updated in place."""
    import torch
    from sources_b200 import learn
    L = 128
    g = torch.Generator(device="cuda").manual_seed(M + inplace)
    E = torch.randn(M, L, device="cuda", generator=g).to(torch.bfloat16)
    EF0 = torch.randn(M, L, device="cuda", generator=g)
    We = (torch.randn(L, L, device="cuda", generator=g) / L ** 0.5).to(torch.bfloat16)
    W2 = (torch.randn(L, L, device="cuda", generator=g) / L ** 0.5).to(torch.bfloat16)
    be = torch.randn(L, device="cuda", generator=g)
    b2 = torch.randn(L, device="cuda", generator=g)
    nodes = max(M // 20, 7)
    P = torch.randn(nodes, 2 * L, device="cuda", generator=g)
    nedge = M - 37 if M > 128 else M
    src = torch.randint(0, nodes, (M,), device="cuda", generator=g, dtype=torch.int32)
    dst = torch.sort(torch.randint(0, nodes, (M,), device="cuda", generator=g, dtype=torch.int32)).values
    # the two-GEMM path
    a = torch.zeros(M, L, device="cuda", dtype=torch.bfloat16)
    e1 = learn.GemmEpi(mode=learn.EPI_EDGE, relu=1, bias=be.data_ptr(), z=None, h=a.data_ptr(), P=P.data_ptr(),
                       src=src.data_ptr(), dst=dst.data_ptr(), nedge=nedge)
    _ws(lib, E, We, M, L, L, e1)
    EF_ref = EF0.clone()
    Eout_ref = torch.zeros(M, L, device="cuda", dtype=torch.bfloat16)
    e2 = learn.GemmEpi(mode=learn.EPI_RESID, bias=b2.data_ptr(), z=EF_ref.data_ptr(), h=Eout_ref.data_ptr())
    _ws(lib, a, W2, M, L, L, e2)
    # fused
    EF = EF0.clone()
    Ein = E.clone()
    Eout = Ein if inplace else torch.zeros(M, L, device="cuda", dtype=torch.bfloat16)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.sphg_gnn_edge_layer(Ein.data_ptr(), EF.data_ptr(), Eout.data_ptr(), P.data_ptr(), src.data_ptr(),
                                 dst.data_ptr(), nedge, M, We.data_ptr(), be.data_ptr(), W2.data_ptr(), b2.data_ptr(),
                                 err.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rc == 0 and int(err.item()) == 0
    assert torch.equal(EF, EF_ref)
    assert torch.equal(Eout, Eout_ref)
    # and against the fp32 arithmetic of the same bf16 operands
    ref_a = E.float() @ We.float().T + be
    ref_a[:nedge] += P[src[:nedge].long(), :L] + P[dst[:nedge].long(), L:]
    ref = EF0 + ref_a.clamp_min(0).to(torch.bfloat16).float() @ W2.float().T + b2
    assert float((EF - ref).abs().max()) <= 2e-2 * float(ref.abs().max())


def test_fused_edge_layer_rejects_bad_arguments(lib):
    import ctypes
    one = ctypes.c_void_p(256)
    odd = ctypes.c_void_p(260)
    assert lib.sphg_gnn_edge_layer(one, one, one, one, one, one, 100, 100, one, one, one, one, one, None) != 0  # M % 128
    assert lib.sphg_gnn_edge_layer(one, one, one, one, one, one, 200, 128, one, one, one, one, one, None) != 0  # nedge > M
    assert lib.sphg_gnn_edge_layer(odd, one, one, one, one, one, 128, 128, one, one, one, one, one, None) != 0  # alignment
    assert lib.sphg_gnn_edge_layer(None, one, one, one, one, one, 128, 128, one, one, one, one, one, None) != 0


@pytest.mark.parametrize("M", [128 * 3, 128 * 1201])
def test_fused_edge_layer_bf16_residual(cuda_ok, lib, M):
    """Without the fp32 residual rows the fused layer keeps the edge latent
    in bf16 alone: Eout = bf16(E + a W2^T + b2), the same bits as the RESID
    epilogue given z = fp32(E); in place, padding rows included."""
    import torch
    from sources_b200 import learn
    L = 128
    g = torch.Generator(device="cuda").manual_seed(M + 5)
    E = torch.randn(M, L, device="cuda", generator=g).to(torch.bfloat16)
    We = (torch.randn(L, L, device="cuda", generator=g) / L ** 0.5).to(torch.bfloat16)
    W2 = (torch.randn(L, L, device="cuda", generator=g) / L ** 0.5).to(torch.bfloat16)
    be = torch.randn(L, device="cuda", generator=g)
    b2 = torch.randn(L, device="cuda", generator=g)
    nodes = max(M // 20, 7)
    P = torch.randn(nodes, 2 * L, device="cuda", generator=g)
    nedge = M - 51
    src = torch.randint(0, nodes, (M,), device="cuda", generator=g, dtype=torch.int32)
    dst = torch.sort(torch.randint(0, nodes, (M,), device="cuda", generator=g, dtype=torch.int32)).values
    a = torch.zeros(M, L, device="cuda", dtype=torch.bfloat16)
    _ws(lib, E, We, M, L, L, learn.GemmEpi(mode=learn.EPI_EDGE, relu=1, bias=be.data_ptr(), z=None, h=a.data_ptr(),
                                           P=P.data_ptr(), src=src.data_ptr(), dst=dst.data_ptr(), nedge=nedge))
    z = E.float()
    Eout_ref = torch.zeros(M, L, device="cuda", dtype=torch.bfloat16)
    _ws(lib, a, W2, M, L, L, learn.GemmEpi(mode=learn.EPI_RESID, bias=b2.data_ptr(), z=z.data_ptr(),
                                           h=Eout_ref.data_ptr()))
    Ein = E.clone()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.sphg_gnn_edge_layer(Ein.data_ptr(), None, Ein.data_ptr(), P.data_ptr(), src.data_ptr(), dst.data_ptr(),
                                 nedge, M, We.data_ptr(), be.data_ptr(), W2.data_ptr(), b2.data_ptr(), err.data_ptr(),
                                 torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rc == 0 and int(err.item()) == 0
    assert torch.equal(Ein, Eout_ref)


def test_segsum_bf16_matches_fp32_rows(cuda_ok, lib):
    """sphg_gnn_segsum_bf16 sums the same rows as sphg_gnn_segsum given their
    fp32 values: identical results."""
    import torch
    L, n = 128, 1000
    g = torch.Generator(device="cuda").manual_seed(3)
    deg = torch.randint(0, 40, (n,), device="cuda", generator=g)
    off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    off[1:] = torch.cumsum(deg, 0)
    E = int(off[-1].item())
    e = torch.randn(E, L, device="cuda", generator=g).to(torch.bfloat16)
    a32 = torch.zeros(n, L, device="cuda")
    a16 = torch.zeros(n, L, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    ef = e.float().contiguous()
    assert lib.sphg_gnn_segsum(ef.data_ptr(), off.data_ptr(), a32.data_ptr(), n, L, 0.0625, s) == 0
    assert lib.sphg_gnn_segsum_bf16(e.data_ptr(), off.data_ptr(), a16.data_ptr(), n, L, 0.0625, s) == 0
    torch.cuda.synchronize()
    assert torch.equal(a32, a16)


@pytest.mark.parametrize("M,inplace", [(128 * 3, True), (128 * 1201, True), (128 * 1201, False)])
def test_edge_layer_nodes_matches_fp32_reference(cuda_ok, lib, M, inplace):
    """sphg_gnn_edge_layer_nodes (sender node rows gathered into the first
    GEMM, K = 256; receiver rows Pd = H Wd^T added in the epilogue) against the
    fp32 arithmetic of the same bf16 operands, and against the projected-row
    kernel (sphg_gnn_edge_layer with P = [H Ws^T | Pd]): the two differ only
    where the rounding of the fp32 sums moves a bf16 hidden or output value by
    one unit; rows beyond nedge use zero node terms; E may be updated in
    place."""
    import torch
    L = 128
    g = torch.Generator(device="cuda").manual_seed(M + 11)
    E = torch.randn(M, L, device="cuda", generator=g).to(torch.bfloat16)
    We = (torch.randn(L, L, device="cuda", generator=g) / L ** 0.5).to(torch.bfloat16)
    Wsd = (torch.randn(2 * L, L, device="cuda", generator=g) / L ** 0.5).to(torch.bfloat16)
    W2 = (torch.randn(L, L, device="cuda", generator=g) / L ** 0.5).to(torch.bfloat16)
    be = torch.randn(L, device="cuda", generator=g)
    b2 = torch.randn(L, device="cuda", generator=g)
    nodes = max(M // 20, 7)
    H = torch.randn(nodes, L, device="cuda", generator=g).to(torch.bfloat16)
    Pd = (H.float() @ Wsd[L:].float().T).contiguous()
    nedge = M - 37
    src = torch.randint(0, nodes, (M,), device="cuda", generator=g, dtype=torch.int32)
    dst = torch.sort(torch.randint(0, nodes, (M,), device="cuda", generator=g, dtype=torch.int32)).values
    s = torch.cuda.current_stream().cuda_stream
    Ein = E.clone()
    Eout = Ein if inplace else torch.zeros(M, L, device="cuda", dtype=torch.bfloat16)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.sphg_gnn_edge_layer_nodes(Ein.data_ptr(), Eout.data_ptr(), H.data_ptr(), Pd.data_ptr(), nodes,
                                       src.data_ptr(), dst.data_ptr(), nedge, M, We.data_ptr(), Wsd.data_ptr(),
                                       be.data_ptr(), W2.data_ptr(), b2.data_ptr(), err.data_ptr(), s)
    torch.cuda.synchronize()
    assert rc == 0 and int(err.item()) == 0
    if not inplace:
        assert torch.equal(Ein, E)
    # fp32 arithmetic of the same bf16 operands
    z = E.float() @ We.float().T + be
    sl, dl = src[:nedge].long(), dst[:nedge].long()
    z[:nedge] += H[sl].float() @ Wsd[:L].float().T + Pd[dl]
    hid = z.clamp_min(0).to(torch.bfloat16).float()
    ref = E.float() + (hid @ W2.float().T + b2)
    out = Eout.float()
    scale = float(ref.abs().max())
    assert float((out - ref).abs().max()) <= 2e-2 * scale
    assert float((out - ref).abs().mean()) <= 2e-3 * float(ref.abs().mean())
    # the projected-row kernel on the same inputs
    P = torch.cat([H.float() @ Wsd[:L].float().T, Pd], dim=1).contiguous()
    Ep = E.clone()
    assert lib.sphg_gnn_edge_layer(Ep.data_ptr(), None, Ep.data_ptr(), P.data_ptr(), src.data_ptr(), dst.data_ptr(),
                                   nedge, M, We.data_ptr(), be.data_ptr(), W2.data_ptr(), b2.data_ptr(),
                                   err.data_ptr(), s) == 0
    torch.cuda.synchronize()
    d = (Ep.float() - out).abs()
    assert float(d.max()) <= 2e-2 * scale
    assert float((d > 0).float().mean()) <= 0.05   # most outputs carry the same bits


def test_edge_layer_nodes_flags_bad_indices_and_arguments(cuda_ok, lib):
    """A sender or receiver index outside [0, nnode) sets bit 1 of *err and
    takes that node term as zero; bad shapes, null or misaligned pointers are
    refused before any launch."""
    import ctypes
    import torch
    L, M, nodes = 128, 256, 40
    g = torch.Generator(device="cuda").manual_seed(3)
    E = torch.randn(M, L, device="cuda", generator=g).to(torch.bfloat16)
    We = (torch.randn(L, L, device="cuda", generator=g) / L ** 0.5).to(torch.bfloat16)
    Ws = (torch.randn(L, L, device="cuda", generator=g) / L ** 0.5).to(torch.bfloat16)
    W2 = (torch.randn(L, L, device="cuda", generator=g) / L ** 0.5).to(torch.bfloat16)
    be = torch.randn(L, device="cuda", generator=g)
    b2 = torch.randn(L, device="cuda", generator=g)
    H = torch.randn(nodes, L, device="cuda", generator=g).to(torch.bfloat16)
    Pd = torch.randn(nodes, L, device="cuda", generator=g)
    src = torch.randint(0, nodes, (M,), device="cuda", generator=g, dtype=torch.int32)
    dst = torch.sort(torch.randint(0, nodes, (M,), device="cuda", generator=g, dtype=torch.int32)).values
    src[5] = nodes          # outside the node rows
    dst[9] = -1
    # the same graph over [zero row | H] and [zero row | Pd]: those terms come from the zero rows
    H2 = torch.cat([torch.zeros(1, L, device="cuda", dtype=torch.bfloat16), H])
    Pd2 = torch.cat([torch.zeros(1, L, device="cuda"), Pd])
    src2, dst2 = src + 1, dst + 1
    src2[5] = 0
    dst2[9] = 0
    s = torch.cuda.current_stream().cuda_stream
    outs = []
    for Hx, Px, sx, dx, n in ((H, Pd, src, dst, nodes), (H2, Pd2, src2, dst2, nodes + 1)):
        Eo = torch.zeros_like(E)
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        assert lib.sphg_gnn_edge_layer_nodes(E.data_ptr(), Eo.data_ptr(), Hx.data_ptr(), Px.data_ptr(), n,
                                             sx.data_ptr(), dx.data_ptr(), M, M, We.data_ptr(), Ws.data_ptr(),
                                             be.data_ptr(), W2.data_ptr(), b2.data_ptr(), err.data_ptr(), s) == 0
        torch.cuda.synchronize()
        outs.append((Eo, int(err.item())))
    assert outs[0][1] == 2 and outs[1][1] == 0
    assert torch.equal(outs[0][0], outs[1][0])
    one = ctypes.c_void_p(256)
    odd = ctypes.c_void_p(260)
    f = lib.sphg_gnn_edge_layer_nodes
    assert f(one, one, one, one, 8, one, one, 100, 100, one, one, one, one, one, one, None) != 0   # M % 128
    assert f(one, one, one, one, 8, one, one, 200, 128, one, one, one, one, one, one, None) != 0   # nedge > M
    assert f(one, one, one, one, 0, one, one, 128, 128, one, one, one, one, one, one, None) != 0   # no nodes
    assert f(odd, one, one, one, 8, one, one, 128, 128, one, one, one, one, one, one, None) != 0   # alignment
    assert f(one, one, one, None, 8, one, one, 128, 128, one, one, one, one, one, one, None) != 0


@pytest.mark.parametrize("M", [128 * 3, 128 * 1201])
def test_edge_encoder_equals_two_gemms(cuda_ok, lib, M):
    """sphg_gnn_edge_encoder (both encoder GEMMs in one kernel, the hidden
    rows kept in TMEM) gives the same bits as two weight-stationary GEMMs with
    the BIAS_ACT epilogue (ReLU, then none)."""
    import ctypes
    import torch
    from sources_b200 import learn
    L, F = 128, 64
    g = torch.Generator(device="cuda").manual_seed(M + 17)
    X = torch.randn(M, F, device="cuda", generator=g).to(torch.bfloat16)
    W1 = (torch.randn(L, F, device="cuda", generator=g) / F ** 0.5).to(torch.bfloat16)
    W2 = (torch.randn(L, L, device="cuda", generator=g) / L ** 0.5).to(torch.bfloat16)
    b1 = torch.randn(L, device="cuda", generator=g)
    b2 = torch.randn(L, device="cuda", generator=g)
    a = torch.zeros(M, L, device="cuda", dtype=torch.bfloat16)
    ref = torch.zeros(M, L, device="cuda", dtype=torch.bfloat16)
    _ws(lib, X, W1, M, L, F, learn.GemmEpi(mode=learn.EPI_BIAS_ACT, relu=1, bias=b1.data_ptr(), h=a.data_ptr()))
    _ws(lib, a, W2, M, L, L, learn.GemmEpi(mode=learn.EPI_BIAS_ACT, relu=0, bias=b2.data_ptr(), h=ref.data_ptr()))
    out = torch.zeros(M, L, device="cuda", dtype=torch.bfloat16)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.sphg_gnn_edge_encoder(X.data_ptr(), out.data_ptr(), M, W1.data_ptr(), b1.data_ptr(), W2.data_ptr(),
                                   b2.data_ptr(), err.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rc == 0 and int(err.item()) == 0
    assert torch.equal(out, ref)
    one, odd = ctypes.c_void_p(256), ctypes.c_void_p(272)
    f = lib.sphg_gnn_edge_encoder
    assert f(one, one, 100, one, one, one, one, one, None) != 0   # M % 128
    assert f(one, odd, 128, one, one, one, one, one, None) != 0   # E_out alignment
    assert f(None, one, 128, one, one, one, one, one, None) != 0


def test_segsum_cat_equals_segsum_and_concat(cuda_ok, lib):
    """sphg_gnn_segsum_cat gives the same bits as sphg_gnn_segsum_bf16 followed
    by sphg_gnn_node_concat, padding rows (zero sums) and nodes without edges
    included."""
    import torch
    L, n, npad = 128, 1000, 1024
    g = torch.Generator(device="cuda").manual_seed(7)
    deg = torch.randint(0, 40, (n,), device="cuda", generator=g)
    deg[::9] = 0
    off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    off[1:] = torch.cumsum(deg, 0)
    E = int(deg.sum())
    e = torch.randn(E, L, device="cuda", generator=g).to(torch.bfloat16)
    h = torch.randn(npad, L, device="cuda", generator=g).to(torch.bfloat16)
    s = torch.cuda.current_stream().cuda_stream
    agg = torch.zeros(npad, L, device="cuda")
    ref = torch.empty(npad, 2 * L, device="cuda", dtype=torch.bfloat16)
    assert lib.sphg_gnn_segsum_bf16(e.data_ptr(), off.data_ptr(), agg.data_ptr(), n, L, 0.0625, s) == 0
    assert lib.sphg_gnn_node_concat(h.data_ptr(), agg.data_ptr(), ref.data_ptr(), npad, L, s) == 0
    out = torch.full((npad, 2 * L), float("nan"), device="cuda").to(torch.bfloat16)
    assert lib.sphg_gnn_segsum_cat(e.data_ptr(), off.data_ptr(), h.data_ptr(), out.data_ptr(), n, npad, L, 0.0625, s) == 0
    torch.cuda.synchronize()
    assert torch.equal(out, ref)


@pytest.mark.parametrize("M", [128 * 2, 128 * 900])
def test_node_mlp_equals_two_gemms(cuda_ok, lib, M):
    """sphg_gnn_node_mlp (both node-MLP GEMMs in one kernel, the hidden rows
    kept in TMEM, the fp32 residual stream updated in place) gives the same bits
    as the weight-stationary GEMMs with the BIAS_ACT (ReLU) and RESID epilogues."""
    import torch
    from sources_b200 import learn
    L = 128
    g = torch.Generator(device="cuda").manual_seed(M + 29)
    X = torch.randn(M, 2 * L, device="cuda", generator=g).to(torch.bfloat16)
    V1 = (torch.randn(L, 2 * L, device="cuda", generator=g) / 16).to(torch.bfloat16)
    V2 = (torch.randn(L, L, device="cuda", generator=g) / L ** 0.5).to(torch.bfloat16)
    c1 = torch.randn(L, device="cuda", generator=g)
    c2 = torch.randn(L, device="cuda", generator=g)
    Z0 = torch.randn(M, L, device="cuda", generator=g)
    ya = torch.zeros(M, L, device="cuda", dtype=torch.bfloat16)
    Zr, hr = Z0.clone(), torch.zeros(M, L, device="cuda", dtype=torch.bfloat16)
    _ws(lib, X, V1, M, L, 2 * L, learn.GemmEpi(mode=learn.EPI_BIAS_ACT, relu=1, bias=c1.data_ptr(), h=ya.data_ptr()))
    _ws(lib, ya, V2, M, L, L, learn.GemmEpi(mode=learn.EPI_RESID, bias=c2.data_ptr(), z=Zr.data_ptr(),
                                            h=hr.data_ptr()))
    Z, h = Z0.clone(), torch.zeros(M, L, device="cuda", dtype=torch.bfloat16)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.sphg_gnn_node_mlp(X.data_ptr(), M, V1.data_ptr(), c1.data_ptr(), V2.data_ptr(), c2.data_ptr(),
                               Z.data_ptr(), h.data_ptr(), err.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rc == 0 and int(err.item()) == 0
    assert torch.equal(Z, Zr)
    assert torch.equal(h, hr)
