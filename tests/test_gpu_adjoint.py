"""The adjoint (mtx_extract_backward) against the oracle's FP64 adjoint and
against FP64 central finite differences of a loss on the torus field.

The loss is the one of the differentiation workload: the mean over vertices
of (|v - c| - 0.35)^2 with v in [0, 1] coordinates of the 512^3 volume and
c = (0.5, 0.5, 0.5).  Finite differences hold the topology fixed (the
active-block list is kept and voxels within 4h of the isovalue, whose
perturbation could flip a cell, are skipped); they are central differences
at h = 1e-4 and h / 2 combined by Richardson extrapolation, whose error is
O(h^4) (a plain central difference has a relative error of about
(h / (f(b) - f(a)))^2, several 1e-3 for this field's edge differences).
"""
import numpy as np
import pytest
import torch

from helpers import blob_volume, mid_iso, to_cuda, u32

pytestmark = pytest.mark.gpu

N_FULL = 512
CROP = (slice(224, 288), slice(224, 288), slice(428, 492))  # z, y, x: a piece of the tube wall


class IsoSurface(torch.autograd.Function):
    """Vertices of the plain extraction as a differentiable function of the
    field and the isovalue (voxel frame, float32 [V, 3])."""

    @staticmethod
    def forward(fctx, field, iso, mctx, block, mode):
        from meshtrex_b200 import api
        vol = api.wrap_volume(field)
        pc = api.push_constants((field.shape[2], field.shape[1], field.shape[0]), block, float(iso.item()))
        mm = api.compute_min_max_mip(mctx, vol, pc)
        f = api.filter_active_blocks(mctx, mm, pc)
        api.read_active_block_count(mctx, f)
        x = api.extract_meshlet_descriptors(mctx, mm, f, pc)
        verts = x.vertices()
        fctx.state = (mctx, vol, pc, mm, f, x, mode, field)
        return verts

    @staticmethod
    def backward(fctx, gv):
        from meshtrex_b200 import api
        mctx, vol, pc, mm, f, x, mode, _ = fctx.state
        dfield, diso = api.extract_backward(mctx, vol, pc, f, x.out.meshletDescriptorBuffer.ptr, x.vertex_count,
                                            gv.float(), mode=mode)
        mctx.synchronize()
        x.free()
        f.free()
        mm.free()
        return dfield, diso.reshape(()), None, None, None


def _forward(ctx, a, block, iso):
    from meshtrex_b200 import api
    vol_t = to_cuda(a)
    vol = api.wrap_volume(vol_t)
    pc = api.push_constants((a.shape[2], a.shape[1], a.shape[0]), block, iso)
    mm = api.compute_min_max_mip(ctx, vol, pc)
    f = api.filter_active_blocks(ctx, mm, pc)
    api.read_active_block_count(ctx, f)
    x = api.extract_meshlet_descriptors(ctx, mm, f, pc)
    return vol_t, vol, pc, mm, f, x


def _free(*objs):
    for o in objs:
        o.free()


@pytest.mark.parametrize("dtype,block", [(np.float32, 8), (np.uint16, 4), (np.uint8, 16), (np.float32, 3)])
@pytest.mark.parametrize("mode", [0, 1])
def test_adjoint_matches_oracle(ctx, oracle, dtype, block, mode):
    from meshtrex_b200 import api
    a = blob_volume((40, 36, 48), dtype, seed=7 + block)
    iso = mid_iso(a)
    vol_t, vol, pc, mm, f, x = _forward(ctx, a, block, iso)
    ids = u32(f.ids())
    V = x.vertex_count
    assert V > 100
    rng = np.random.default_rng(block)
    g = rng.standard_normal((V, 3)).astype(np.float32)
    dfield, diso = api.extract_backward(ctx, vol, pc, f, x.out.meshletDescriptorBuffer.ptr, V,
                                        torch.from_numpy(g).cuda(), mode=mode)
    ctx.synchronize()
    ref, ref_iso = oracle.mc_adjoint(a, block, iso, ids, g)
    got = dfield.cpu().numpy().astype(np.float64)
    scale = np.abs(ref).max()
    assert scale > 0
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6 * scale)
    assert abs(float(diso.item()) - ref_iso) <= 1e-5 * max(abs(ref_iso), 1e-3 * scale)
    _free(x, f, mm)


def test_ndc_frame_and_vertex_data_stride(ctx, oracle):
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    a = blob_volume((32, 40, 24), np.float32, seed=3)
    iso = mid_iso(a)
    vol_t, vol, pc, mm, f, x = _forward(ctx, a, 8, iso)
    V = x.vertex_count
    rng = np.random.default_rng(5)
    g8 = rng.standard_normal((V, 8)).astype(np.float32)  # VertexData layout: position gradient first
    dfield, diso = api.extract_backward(ctx, vol, pc, f, x.out.meshletDescriptorBuffer.ptr, V,
                                        torch.from_numpy(g8).cuda(), frame=L.FRAME_NDC)
    ctx.synchronize()
    dims = np.array([a.shape[2], a.shape[1], a.shape[0]], np.float32)
    g_voxel = (g8[:, :3] * (np.float32(2.0) / dims)).astype(np.float32)
    ref, ref_iso = oracle.mc_adjoint(a, 8, iso, u32(f.ids()), g_voxel)
    scale = np.abs(ref).max()
    np.testing.assert_allclose(dfield.cpu().numpy(), ref, rtol=1e-5, atol=1e-6 * scale)
    assert abs(float(diso.item()) - ref_iso) <= 1e-5 * max(abs(ref_iso), 1e-3 * scale)
    _free(x, f, mm)


def test_deterministic_mode_is_bitwise_reproducible(ctx):
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    a = blob_volume((48, 48, 48), np.uint16, seed=17)
    iso = mid_iso(a)
    vol_t, vol, pc, mm, f, x = _forward(ctx, a, 8, iso)
    V = x.vertex_count
    g = torch.randn((V, 3), generator=torch.Generator().manual_seed(1)).cuda()
    runs = [api.extract_backward(ctx, vol, pc, f, x.out.meshletDescriptorBuffer.ptr, V, g,
                                 mode=L.ADJOINT_DETERMINISTIC) for _ in range(3)]
    atomic = api.extract_backward(ctx, vol, pc, f, x.out.meshletDescriptorBuffer.ptr, V, g)
    ctx.synchronize()
    for d, i in runs[1:]:
        assert torch.equal(d.view(torch.int32), runs[0][0].view(torch.int32))
        assert torch.equal(i.view(torch.int32), runs[0][1].view(torch.int32))
    torch.testing.assert_close(atomic[0], runs[0][0], rtol=1e-5, atol=1e-6 * float(atomic[0].abs().max()))
    assert torch.equal(atomic[1], runs[0][1])  # dL/diso is reduced in a fixed order in both modes
    _free(x, f, mm)


def test_topology_change_is_reported(ctx):
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api
    a = blob_volume((32, 32, 32), np.float32, seed=23)
    iso = mid_iso(a)
    vol_t, vol, pc, mm, f, x = _forward(ctx, a, 8, iso)
    V = x.vertex_count
    ctx.synchronize()
    vol_t.neg_()  # a different field under the same forward outputs
    api.extract_backward(ctx, vol, pc, f, x.out.meshletDescriptorBuffer.ptr, V,
                         torch.zeros((V, 3), device="cuda"))
    with pytest.raises(L.MtxError) as e:
        ctx.synchronize()
    assert e.value.status == 8  # MTX_ERR_INTERNAL
    _free(x, f, mm)


def _loss64(field64, block, iso, ids, offset_xyz):
    from oracle import oracle as O
    m = O.mc_extract(field64, block, iso, ids, want_xyz=False, want_xyz64=True, want_indices=False)
    v = (m.xyz64 + offset_xyz) / (N_FULL - 1)
    return np.mean((np.linalg.norm(v - 0.5, axis=1) - 0.35) ** 2)


def _torus_loss(v, offset_xyz):
    vn = (v + torch.tensor(offset_xyz, dtype=torch.float32, device=v.device)) / (N_FULL - 1)
    return ((vn - 0.5).norm(dim=1) - 0.35).pow(2).mean()


def _richardson(fn, x0, h):
    d1 = (fn(x0 + h) - fn(x0 - h)) / (2 * h)
    d2 = (fn(x0 + h / 2) - fn(x0 - h / 2)) / h
    return (4 * d2 - d1) / 3, d1


@pytest.mark.parametrize("mode", [0, 1])
def test_autograd_on_torus_crop_matches_finite_differences(ctx, oracle, mode):
    from meshtrex_b200 import synth
    full = synth.torus(N_FULL, seed=4, device="cuda")
    crop = full[CROP].contiguous()
    del full
    offset = np.array([CROP[2].start, CROP[1].start, CROP[0].start], np.float64)
    block, iso = 8, 0.0
    field = crop.clone().requires_grad_(True)
    iso_t = torch.tensor(iso, device="cuda", requires_grad=True)
    v = IsoSurface.apply(field, iso_t, ctx, block, mode)
    assert v.shape[0] > 1000
    _torus_loss(v, offset).backward()
    g = field.grad.cpu().numpy().astype(np.float64)
    g_iso = float(iso_t.grad.item())

    f32 = crop.cpu().numpy()
    f64 = f32.astype(np.float64)
    ids = oracle.compact(oracle.minmax_halo(f32, block), oracle.F32, iso)
    # the CPU reference gradient for the same dL/dvertex
    v_det = v.detach().requires_grad_(True)
    (gv,) = torch.autograd.grad(_torus_loss(v_det, offset), [v_det])
    ref, ref_iso = oracle.mc_adjoint(f32, block, iso, ids, gv.cpu().numpy().astype(np.float32))
    np.testing.assert_allclose(g, ref, rtol=1e-5, atol=1e-6 * np.abs(ref).max())
    assert abs(g_iso - ref_iso) <= 1e-5 * abs(ref_iso)

    h = 1e-4
    rng = np.random.default_rng(4)
    support = np.argwhere(np.abs(g) > 0)
    picks = [tuple(p) for p in support[rng.choice(len(support), 100, replace=False)]]
    picks += [tuple(int(rng.integers(0, s)) for s in f32.shape) for _ in range(100)]
    gmax = np.abs(g).max()
    checked = 0
    for zyx in picks:
        if abs(f64[zyx] - iso) < 4 * h:
            continue

        def fn(val, zyx=zyx):
            f = f64.copy()
            f[zyx] = val
            return _loss64(f, block, iso, ids, offset)

        fd, fd_plain = _richardson(fn, f64[zyx], h)
        assert abs(fd - g[zyx]) <= 1e-4 * max(abs(fd), 1e-3 * gmax), (zyx, fd, g[zyx], fd_plain)
        checked += 1
    assert checked >= 150

    # Shifting the isovalue moves every vertex at once; it keeps the topology
    # only while no voxel crosses it, so its step stays below the smallest
    # distance of a voxel to the isovalue.
    gap = float(np.abs(f64 - iso).min())
    assert gap > 0
    h_iso = min(h, gap / 4)

    def fn_iso(s):
        return _loss64(f64 - s, block, iso, ids, offset)  # iso + s <=> field - s

    fd_iso, _ = _richardson(fn_iso, 0.0, h_iso)
    assert abs(fd_iso - g_iso) <= 1e-4 * abs(fd_iso)
    # each edge's two field terms sum to minus its isovalue term
    assert abs(g.sum() + g_iso) <= 1e-4 * abs(g_iso)
