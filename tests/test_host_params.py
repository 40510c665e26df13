"""The host mirror's parameter defaults and option names are the reference's,
so a caller that switches backends gets the same stack from the same settings,
and a misspelt option is an error rather than another option. CPU only."""
import pytest

import lapstack_b200 as L
from lapstack_b200 import _lib


def test_fuse_defaults_are_the_reference_defaults():
    # fuse.rs:94-107: levels None (auto), energy radius 1, DevEntropy top rule of radius 2 over 256 bins,
    # no chroma, depth level 2, halo control off
    p = L.FuseParams()
    assert (p.levels, p.energy_radius, p.top_rule, p.top_radius, p.entropy_bins, p.use_chroma, p.depth_level,
            p.halo) == (0, 1, "de", 2, 256, False, 2, 0.0)
    c = p.c()
    assert (c.levels, c.energy_radius, c.top_rule, c.top_radius, c.entropy_bins, c.use_chroma, c.depth_level) == \
        (0, 1, 0, 2, 256, 0, 2)


def test_align_defaults_are_the_reference_defaults():
    # align.rs:66-70: shift, scale and rotation free, similarity model (align.rs:88), no coarsening,
    # Spline4x4 interpolation (align.rs:137)
    p = L.AlignParams()
    assert (p.shift, p.scale, p.rotation, p.model, p.coarsen, p.interp) == (True, True, True, "similarity", 0, "spline4x4")
    assert p.free() == [True, True, True, True, False, False, False, False]
    c = p.c()
    assert (c.enabled, c.shift, c.scale, c.rotation, c.model, c.coarsen, c.host_search) == (1, 1, 1, 1, 0, 0, 0)
    assert L.engine.INTERPS[c.interp] == "spline4x4"


def test_depth_defaults_are_the_reference_defaults():
    # depth.rs:93-109: scale 1, RDF focus r_in 1 / r_out 3, aggregation radius 3 and eps 1e-4, lambda 3,
    # sigma_c 0.04, 200 CG iterations, median on, guided upsampling radius 2 eps 1e-2, gate 1, robust 1
    p = L.DepthParams()
    assert (p.scale, p.focus, p.r_in, p.r_out, p.agg_radius, p.agg_eps, p.lam, p.sigma_c, p.cg_iters, p.median,
            p.upsample, p.up_radius, p.up_eps, p.gate, p.robust) == \
        (1, "rdf", 1, 3, 3, 1e-4, 3.0, 0.04, 200, True, "guided", 2, 1e-2, 1.0, 1.0)
    # the two switches that leave the reference's formulas are off by default
    assert (p.edge_mode, p.vcycle_mode) == (0, 0)
    c = p.c()
    assert isinstance(c, _lib.DepthParamsC)
    assert (c.enabled, c.focus, c.upsample, c.median) == (1, 0, 1, 1)


def test_option_names_take_the_reference_spellings():
    # fuse.rs:59 TopRule::parse
    for name, code in [("de", 0), ("dev-entropy", 0), ("dev", 1), ("deviation", 1), ("avg", 2), ("average", 2)]:
        assert L.FuseParams(top_rule=name).c().top_rule == code
    # align.rs:95 AlignModel::parse and align.rs:148 Interp::parse trim and lower-case
    for name, code in [("similarity", 0), (" Sim ", 0), ("affine", 1), ("projective", 2), ("perspective", 2),
                       ("HOMOGRAPHY", 2)]:
        assert L.AlignParams(model=name).c().model == code
    assert L.AlignParams(model="sim").free() == L.AlignParams().free()
    assert L.AlignParams(model="homography").free() == [True] * 8
    # align.rs:1208-1209 free_mask
    assert L.AlignParams(rotation=False, model="affine").free() == [True, True, True, False, True, True, False, False]
    assert L.AlignParams(model="projective").free() == [True] * 8
    for name, code in [("nn", 0), ("linear", 1), ("cubic", 2), ("spline16", 3), ("Spline4x4", 3), ("spline36", 4),
                       ("lanczos", 5)]:
        assert L.AlignParams(interp=name).c().interp == code
    assert (L.DepthParams(focus="sml").c().focus, L.DepthParams(upsample="bilinear").c().upsample) == (1, 0)


@pytest.mark.parametrize("make", [lambda: L.FuseParams(top_rule="entropy").c(),
                                  lambda: L.AlignParams(model="rigid").c(),
                                  lambda: L.AlignParams(model="rigid").free(),
                                  lambda: L.AlignParams(interp="spline8x8").c(),
                                  lambda: L.DepthParams(focus="laplacian").c(),
                                  lambda: L.DepthParams(upsample="nearest").c(),
                                  lambda: L.DepthParams(upsample="Guided").c()])
def test_unknown_option_names_are_errors(make):
    """An unknown name is refused (the reference's parsers return None), never mapped to another option."""
    with pytest.raises(L.LsbError, match="unknown"):
        make()


def c_check(fp=None, ap=None, dp=None):
    """lsb_check_params on raw C structs (codes the Python names cannot produce); None or the error text."""
    import ctypes as C
    lib = L.load()
    err = lib.lsb_check_params(C.byref(fp or L.FuseParams().c()), C.byref(ap or L.AlignParams().c()),
                               C.byref(dp or L.DepthParams().c()))
    if not err:
        return None
    msg = C.cast(err, C.c_char_p).value.decode()
    lib.lsb_free_str(err)
    return msg


def test_check_params_accepts_the_defaults_without_a_device():
    L.check_params()
    L.check_params(L.FuseParams(), L.AlignParams(), L.DepthParams())
    L.check_params(L.FuseParams(energy_radius=2, top_rule="avg", top_radius=4),
                   L.AlignParams(model="projective", interp="lanczos3"),
                   L.DepthParams(focus="sml", sml_step=3, scale=2, agg_radius=19, upsample="bilinear", edge_mode=1,
                                 vcycle_mode=1))
    assert c_check() is None


def with_field(struct, **kw):
    for k, v in kw.items():
        setattr(struct, k, v)
    return struct


@pytest.mark.parametrize("field,value,text", [
    ("energy_radius", 3, "energy_radius"), ("top_rule", 3, "top_rule"), ("top_radius", 5, "top_radius")])
def test_check_params_refuses_fuse_codes_out_of_range(field, value, text):
    assert text in c_check(fp=with_field(L.FuseParams().c(), **{field: value}))


@pytest.mark.parametrize("field,value,text", [("model", 3, "model"), ("interp", 6, "interp")])
def test_check_params_refuses_align_codes_out_of_range(field, value, text):
    assert text in c_check(ap=with_field(L.AlignParams().c(), **{field: value}))
    # a disabled pass is not checked
    assert c_check(ap=with_field(L.AlignParams().c(enabled=False), **{field: value})) is None


@pytest.mark.parametrize("fields,text", [
    ({"scale": 3}, "scale"), ({"focus": 2}, "focus"), ({"r_in": 3, "r_out": 3}, "rdf radii"),
    ({"r_out": 4}, "rdf radii"), ({"focus": 1, "sml_step": 0}, "sml step"), ({"focus": 1, "sml_step": 4}, "sml step"),
    ({"agg_radius": 20}, "agg_radius"), ({"agg_radius": 40000}, "agg_radius"), ({"agg_radius": 0xFFFFFFFF}, "agg_radius"),
    ({"upsample": 2}, "upsample"), ({"up_radius": (1 << 20) + 1}, "up_radius"), ({"edge_mode": 2}, "edge_mode"),
    ({"vcycle_mode": 2}, "vcycle_mode")])
def test_check_params_refuses_depth_settings_out_of_range(fields, text):
    assert text in c_check(dp=with_field(L.DepthParams().c(), **fields))
    assert c_check(dp=with_field(L.DepthParams().c(enabled=False), **fields)) is None


def test_check_params_largest_aggregation_radius_is_19():
    # the aggregation tile with its halos must fit the 227 KiB of shared memory a CTA can have:
    # 232,192 bytes at radius 19, 247,808 at 20
    assert c_check(dp=with_field(L.DepthParams().c(), agg_radius=19)) is None
    assert c_check(dp=with_field(L.DepthParams().c(), agg_radius=0)) is None
    with pytest.raises(L.LsbError, match="agg_radius"):
        L.check_params(depth=L.DepthParams(agg_radius=20))
