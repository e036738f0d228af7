"""Device-side topology apply and the GPU evaluation renderer through the C
ABI.

Topology: a random plan (kept, pruned, split and duplicated splats, refine
decay, opacity reset) built on the device is bit-identical to the oracle's
restatement of topology/apply.rs, for FP32 and BF16 SH storage; a plan row
naming a missing splat is reported as GSR_ERR_INVALID_ARG.

Evaluation: SplatEvaluationRenderer returns the forward image clamped to
[0, 1] and quantised to 1/255, like the reference's u8 renderer output.
"""
import numpy as np
import pytest

from _parity import oracle_forward
from oracle import oracle as O
from rustscan_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _plan(n, rng):
    rows = []
    for src in range(n):
        r = rng.random()
        if r < 0.15:
            continue  # pruned
        if r < 0.45:
            s = float(rng.normal(0.0, 1.0))
            rows += [(src, 1, s), (src, 2, s)]  # split
        else:
            rows.append((src, 0, 0.0))
    rows += [(int(rng.integers(0, n)), 0, 0.0) for _ in range(n // 10)]  # duplicates
    return rows


@pytest.mark.parametrize("sh_dtype", ["f32", "bf16"])
@pytest.mark.parametrize("opts", [dict(), dict(refine_decay=(0.1, 0.2, 0.3), opacity_reset=True)])
def test_topology_apply_matches_oracle(gsr_ctx_factory, sh_dtype, opts):
    import torch

    from rustscan_b200 import TopologyPlan, apply_topology, host_splats_to_device

    sc = S.small_scene(n=3000, degree=3, seed=130)
    rng = np.random.default_rng(7)
    rows = _plan(sc.n, rng)
    ctx = gsr_ctx_factory(max_splats=sc.n, sh_dtype=sh_dtype)
    dt = torch.bfloat16 if sh_dtype == "bf16" else torch.float32
    splats = host_splats_to_device(sc, sh_dtype=dt)
    out = apply_topology(ctx, splats, TopologyPlan(rows, **opts))
    torch.cuda.synchronize()
    sh_in = splats.sh_coeffs.float().cpu().numpy()
    dec = opts.get("refine_decay")
    t, s, o = O.topology_apply(sc.transforms, sh_in, sc.raw_opacity, rows, has_decay=dec is not None,
                               opacity_decay=dec[0] if dec else 0.0, scale_decay=dec[1] if dec else 0.0,
                               train_t=dec[2] if dec else 0.0, opacity_reset=opts.get("opacity_reset", False))
    assert out.num_splats() == len(rows)
    np.testing.assert_array_equal(out.transforms.cpu().numpy(), t)
    np.testing.assert_array_equal(out.raw_opacities.cpu().numpy(), o)
    assert out.sh_coeffs.dtype == dt
    np.testing.assert_array_equal(out.sh_coeffs.float().cpu().numpy(), s)
    # The source set is untouched.
    np.testing.assert_array_equal(splats.transforms.cpu().numpy(), sc.transforms)


def test_topology_bad_source_is_reported(gsr_ctx_factory):
    from rustscan_b200 import GsrError, TopologyPlan, apply_topology, host_splats_to_device

    sc = S.small_scene(n=100, degree=1, seed=131)
    ctx = gsr_ctx_factory(max_splats=sc.n)
    splats = host_splats_to_device(sc)
    with pytest.raises(GsrError) as ei:
        apply_topology(ctx, splats, TopologyPlan([(0, 0, 0.0), (sc.n + 5, 0, 0.0)]))
    assert ei.value.status == 1
    # The context stays usable afterwards.
    out = apply_topology(ctx, splats, TopologyPlan([(1, 0, 0.0)]))
    assert out.num_splats() == 1


def test_evaluation_renderer_quantises_forward_image():
    from rustscan_b200 import SplatEvaluationRenderer

    sc = S.small_scene(n=2000, degree=2, width=80, height=60, seed=132)
    cam = sc.cameras[0]
    r = SplatEvaluationRenderer(80, 60, max_splats=4096)
    img = r.render(sc, cam)
    o = oracle_forward(sc, cam)
    ref = np.round(np.clip(o.image[..., :3], 0.0, 1.0) * 255.0) / 255.0
    assert img.shape == (80 * 60 * 3,)
    # Values sit on the 1/255 grid; they equal the oracle's except where the
    # image lies within 1e-5 of a rounding boundary.
    np.testing.assert_allclose(img * 255.0, np.round(img * 255.0), atol=1e-3)
    assert np.mean(np.abs(img - ref.reshape(-1)) > 1e-6) < 1e-3
