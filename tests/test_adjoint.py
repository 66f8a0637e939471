"""Path-replay adjoint: gradients against central finite differences of the forward
renderer (common random numbers), plus a torch.autograd wrapper used for a few steps
of texture recovery.

The loss is linear in the image, L = sum_v sum_p w_p . I_v,p, so d_rgb = w.  Finite
differences perturb one parameter by +-h and re-render with the same seed; the adjoint
runs with other seeds.  Both estimates are noisy: each is averaged over several seeds
and the tolerance is the larger of a relative bound and 4 standard errors of the
difference.
"""
from pathlib import Path

import numpy as np
import pytest

import fumeng_b200 as fb
from fumeng_b200 import synth
from fumeng_b200.scene import SceneSpec, camera_struct

pytestmark = pytest.mark.gpu

RES = 48
GOLDEN = Path(__file__).resolve().parent / "golden"


def grad_scene(**kw) -> SceneSpec:
    return synth.gradient_scene(res=RES, **kw)


def weights(seed=0):
    return np.random.default_rng(seed).uniform(0.5, 1.5, (RES, RES, 3)).astype(np.float32)


def loss(scene, spec, w, spp, seed):
    p = spec.render_params(spp=spp, seed=seed)
    img = scene.render(spec.camera_struct(), p, want_aov=False)[0]
    return float((w.astype(np.float64) * img).sum())


def adjoint(ctx, spec, w, spp, seeds, shapes, materials=False):
    sc = ctx.create_scene(spec.to_desc())
    outs = []
    for s in seeds:
        p = spec.render_params(spp=spp, seed=s)
        tg, mg, _, st = sc.render_adjoint([spec.camera_struct()], [p], [w], shapes, material_grads=materials)
        assert st.nan_samples == 0
        outs.append((tg, mg))
    return outs


def mean_sem(x):
    x = np.asarray(x, np.float64)
    return x.mean(0), x.std(0, ddof=1) / np.sqrt(len(x))


def check(name, a, sa, f, sf, rel):
    tol = max(rel * abs(f), 4.0 * np.hypot(sa, sf))
    assert abs(a - f) <= tol, f"{name}: adjoint {a:.6g} +- {sa:.2g} vs FD {f:.6g} +- {sf:.2g}"


@pytest.fixture(scope="module")
def ctx():
    c = fb.Context(0)
    yield c
    c.close()


SPP = 4096
SEEDS_FD = [101, 102, 103, 104]
SEEDS_ADJ = [201, 202, 203, 204]


def test_material_constant_gradients(ctx):
    """d/d{basecolor rgb, metallic, roughness} of a constant Disney material and
    d/d basecolor of a Lambert material."""
    w = weights()
    spec = grad_scene()
    holder = spec.to_desc()
    im = holder.material_index
    outs = adjoint(ctx, spec, w, SPP, SEEDS_ADJ, {}, materials=True)
    mg = np.stack([o[1] for o in outs])
    a_mean, a_sem = mean_sem(mg)
    h = 0.02
    cases = [("probe", 0, "basecolor", 0), ("probe", 1, "basecolor", 1), ("probe", 2, "basecolor", 2),
             ("probe", 3, "metallic", None), ("probe", 4, "roughness", None), ("lam", 0, "basecolor", 0),
             ("lam", 2, "basecolor", 2)]
    for mat, gi, key, ch in cases:
        fds = []
        for s in SEEDS_FD:
            vals = []
            for sign in (1.0, -1.0):
                base = grad_scene()
                m = next(x for x in base.materials if x["name"] == mat)
                if ch is None:
                    m[key] = float(m[key]) + sign * h
                else:
                    v = list(m[key])
                    v[ch] += sign * h
                    m[key] = v
                sc = ctx.create_scene(base.to_desc())
                vals.append(loss(sc, base, w, SPP, s))
                sc.destroy()
            fds.append((vals[0] - vals[1]) / (2 * h))
        f_mean, f_sem = mean_sem(fds)
        i = im[mat]
        check(f"{mat}.{key}[{gi}]", a_mean[i, gi], a_sem[i, gi], f_mean, f_sem, 0.03)


def test_texel_gradients(ctx):
    """d/d texel of the basecolor texture (rgb) and of the roughness (G) / metallic (B)
    texture of the plane's material."""
    w = weights(1)
    spec = grad_scene()
    holder = spec.to_desc()
    ti = holder.texture_index
    shapes = {ti["base"]: (4, 4), ti["rm"]: (4, 4)}
    outs = adjoint(ctx, spec, w, SPP, SEEDS_ADJ, shapes)
    h = 0.03
    sc = ctx.create_scene(holder)
    for tex, texel, ch in [("base", (1, 1), 0), ("base", (2, 2), 1), ("base", (1, 2), 2), ("rm", (1, 2), 1),
                           ("rm", (2, 1), 2), ("rm", (2, 2), 1)]:
        a_mean, a_sem = mean_sem([o[0][ti[tex]][texel + (ch,)] for o in outs])
        orig = spec.textures[tex]
        fds = []
        for s in SEEDS_FD:
            vals = []
            for sign in (1.0, -1.0):
                t = orig.copy()
                t[texel + (ch,)] += sign * h
                sc.update_texture(ti[tex], t)
                vals.append(loss(sc, spec, w, SPP, s))
            fds.append((vals[0] - vals[1]) / (2 * h))
        sc.update_texture(ti[tex], orig)
        f_mean, f_sem = mean_sem(fds)
        check(f"{tex}{texel}[{ch}]", a_mean, a_sem, f_mean, f_sem, 0.03)
    sc.destroy()


def test_env_texel_gradients(ctx):
    """d/d env texel: camera misses, NEE of the environment and MIS rays that escape."""
    w = weights(2)
    spec = grad_scene()
    holder = spec.to_desc()
    ti = holder.texture_index
    sky = spec.textures["sky"]
    outs = adjoint(ctx, spec, w, SPP, SEEDS_ADJ, {ti["sky"]: sky.shape[:2]})
    g = np.stack([o[0][ti["sky"]] for o in outs])
    a_mean_all, _ = mean_sem(g)
    # the texels with the largest gradients (several views of the sky reach them)
    flat = np.argsort(-np.abs(a_mean_all).reshape(-1))[:4]
    sc = ctx.create_scene(holder)
    h = 0.05
    for fi in flat:
        idx = np.unravel_index(fi, a_mean_all.shape)
        a_mean, a_sem = mean_sem(g[(slice(None),) + idx])
        fds = []
        for s in SEEDS_FD:
            vals = []
            for sign in (1.0, -1.0):
                t = sky.copy()
                t[idx] += sign * h * max(1.0, abs(float(sky[idx])))
                sc.update_texture(ti["sky"], t)
                vals.append(loss(sc, spec, w, SPP, s))
            fds.append((vals[0] - vals[1]) / (2 * h * max(1.0, abs(float(sky[idx])))))
        sc.update_texture(ti["sky"], sky)
        f_mean, f_sem = mean_sem(fds)
        check(f"sky{idx}", a_mean, a_sem, f_mean, f_sem, 0.03)
    sc.destroy()


def test_gradients_match_reference_double_fd(ctx):
    """Material-constant gradients against central differences of the reference's double
    build (tests/golden/adj_fd_ref.npz, made by make_golden.py from the same scene and
    loss weights)."""
    g = np.load(GOLDEN / "adj_fd_ref.npz")
    w = np.random.default_rng(int(g["wseed"])).uniform(0.5, 1.5, (RES, RES, 3)).astype(np.float32)
    spec = grad_scene()
    im = spec.to_desc().material_index
    outs = adjoint(ctx, spec, w, SPP, SEEDS_ADJ, {}, materials=True)
    a_mean, a_sem = mean_sem(np.stack([o[1] for o in outs]))
    for ci, name in enumerate(g["cases"]):
        mat, key, ch = str(name).split(".")
        gi = int(ch) if key == "basecolor" else (3 if key == "metallic" else 4)
        f_mean, f_sem = mean_sem(g["fd"][ci])
        check(f"reference {name}", a_mean[im[mat], gi], a_sem[im[mat], gi], f_mean, f_sem, 0.05)


def test_adjoint_image_matches_forward(ctx):
    """The adjoint's primal pass renders the same samples as the forward render."""
    spec = grad_scene()
    sc = ctx.create_scene(spec.to_desc())
    p = spec.render_params(spp=64, seed=9)
    fwd = sc.render(spec.camera_struct(), p, want_aov=False)[0]
    _, _, imgs, _ = sc.render_adjoint([spec.camera_struct()], [p], [weights()], {}, want_image=True)
    np.testing.assert_allclose(imgs[0], fwd, rtol=2e-5, atol=2e-6)
    sc.destroy()


def test_adjoint_zero_weights_give_zero_gradients(ctx):
    spec = grad_scene()
    holder = spec.to_desc()
    ti = holder.texture_index
    sc = ctx.create_scene(holder)
    p = spec.render_params(spp=4, seed=3)
    tg, mg, _, _ = sc.render_adjoint([spec.camera_struct()], [p], [np.zeros((RES, RES, 3), np.float32)],
                                     {ti["base"]: (4, 4), ti["sky"]: (8, 16)}, material_grads=True)
    assert not np.any(tg[ti["base"]]) and not np.any(tg[ti["sky"]]) and not np.any(mg)
    sc.destroy()


def test_adjoint_rejects_megakernel_mode(ctx):
    spec = grad_scene()
    sc = ctx.create_scene(spec.to_desc())
    p = spec.render_params(spp=1, mode=fb.FM_MODE_MEGAKERNEL)
    with pytest.raises(fb.FumengError):
        sc.render_adjoint([spec.camera_struct()], [p], [weights()], {})
    sc.destroy()


# ---- torch.autograd wrapper (test harness only) ----------------------------------------


def test_autograd_texture_recovery(ctx):
    """A few Adam steps on the basecolor / roughness-metallic textures of a small
    inverse-rendering scene lower the L2 image loss against the hidden targets."""
    torch = pytest.importorskip("torch")
    tex_res, res, nviews = 32, 64, 4
    target = synth.inverse_scene(tex_res=tex_res, plane_n=40, sphere_nu=32, sphere_nv=16, res=res, target=True)
    init = synth.inverse_scene(tex_res=tex_res, plane_n=40, sphere_nu=32, sphere_nv=16, res=res, target=False)
    cams = [camera_struct(c) for c in synth.inverse_views(nviews)]
    th = target.to_desc()
    ti = th.texture_index
    tsc = ctx.create_scene(th)
    fwd = [target.render_params(spp=64, seed=1000 + v) for v in range(nviews)]
    ref = np.stack([tsc.render(c, p, want_aov=False)[0] for c, p in zip(cams, fwd)])
    tsc.destroy()
    sc = ctx.create_scene(init.to_desc())
    shapes = {ti["basecolor"]: (tex_res, tex_res), ti["rm"]: (tex_res, tex_res)}

    class RenderViews(torch.autograd.Function):
        @staticmethod
        def forward(fctx, base, rm, it):
            sc.update_texture(ti["basecolor"], base.detach().numpy())
            sc.update_texture(ti["rm"], rm.detach().numpy())
            ps = [init.render_params(spp=16, seed=10 * it + v) for v in range(nviews)]
            fctx.it = it
            return torch.from_numpy(np.stack([sc.render(c, p, want_aov=False)[0] for c, p in zip(cams, ps)]))

        @staticmethod
        def backward(fctx, g):
            ps = [init.render_params(spp=16, seed=777 + 10 * fctx.it + v) for v in range(nviews)]
            tg, _, _, _ = sc.render_adjoint(cams, ps, list(g.numpy().astype(np.float32)), shapes)
            return (torch.from_numpy(tg[ti["basecolor"]]).float(), torch.from_numpy(tg[ti["rm"]]).float(), None)

    base = torch.full((tex_res, tex_res, 3), 0.5, requires_grad=True)
    rm = torch.tensor(init.textures["rm"], requires_grad=True)
    opt = torch.optim.Adam([base, rm], lr=0.03)
    ref_t = torch.from_numpy(ref)
    losses = []
    for it in range(12):
        opt.zero_grad()
        img = RenderViews.apply(base, rm, it)
        L = ((img - ref_t) ** 2).mean()
        L.backward()
        opt.step()
        with torch.no_grad():
            base.clamp_(0.0, 1.0)
            rm.clamp_(0.0, 1.0)
            rm[..., 0] = 0.0
        losses.append(float(L))
    assert losses[-1] < 0.8 * losses[0], losses
    sc.destroy()
