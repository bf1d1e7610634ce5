"""Checkpoint files in the reference's v3 format, on the CPU.

* The oracle restatement (oracle/checkpoint.py) is pinned to the published
  FNV-1a 64 vectors and to the reference's own checkpoint tests
  (crates/lbm-core/src/solver.rs:6296-6700): resume bit-exactness for f32 and
  f64, the mismatch codes and their messages, corrupt / truncated payloads,
  scalar and QOI round trips, stale stash and carried solid moments.
* The library's host writer (lbmb_checkpoint_write_host) produces the same
  bytes as the oracle's writer, manifest and rank file, and its reader
  (lbmb_checkpoint_read_host) returns the oracle's state and the same error
  codes. No device is involved.
"""
import json
import os
import shutil

import numpy as np
import pytest

import lbmflow_b200 as lb
from oracle import checkpoint as ock
from oracle import oracle as o

FNV_VECTORS = [(b"", 0xCBF29CE484222325), (b"a", 0xAF63DC4C8601EC8C), (b"foobar", 0x85944171F73967E8)]


def test_fnv1a64_published_vectors():
    for data, h in FNV_VECTORS:
        assert ock.fnv1a64(data) == h
        assert lb.fnv1a64(data) == h


def channel_case(bits, q=19, collision="trt", scalar_q=7, steps=9):
    """Periodic-x/z channel with a moving top wall, Guo force, a scalar."""
    dims, nu = (8, 7, 6), 0.05
    u = np.zeros(18)
    u[9] = 0.03
    solid, wall = o.wall_rims(dims, [False, False, True, True, False, False], u)
    os_ = 1.0 / (3.0 * nu + 0.5)
    kw = dict(q=q, real_bits=bits, collision=collision, nu=nu, omega_shear=os_, periodic=(True, False, True),
              force=(1e-6, 0.0, 0.0), solid=solid, wall_u=wall)
    s = o.OracleSolver(dims, **kw)
    if scalar_q:
        k = s.scalar_enable(0.02, q=scalar_q)
        s.scalar_set(k, np.where(solid == 0, np.linspace(0.0, 1.0, s.n), 0.0))
    s.step(steps)
    spec = ock.solver_spec(s, collision, nu, lb.MAGIC_STD, os_, (True, False, True), (1e-6, 0.0, 0.0))
    return s, spec, solid, wall, kw


def lib_state(st, names, qoi=None):
    return dict(step=st["step"], f=st["f"], moments=st["moments"], force_field=st["force_field"],
                scalars=[dict(name=nm, diffusivity=x["diffusivity"], q=x["q"], h=x["h"], conc=x["conc"])
                         for nm, x in zip(names, st["scalars"])], qoi=qoi)


def same_bytes(a, b):
    with open(a, "rb") as fa, open(b, "rb") as fb:
        return fa.read() == fb.read()


@pytest.mark.parametrize("bits,q,coll,sq", [(64, 19, "trt", 7), (32, 19, "trt", 19), (64, 27, "cm", 27),
                                            (32, 27, "cm", 7)])
def test_library_writer_is_byte_identical_to_oracle(tmp_path, bits, q, coll, sq):
    s, spec, solid, wall, _ = channel_case(bits, q, coll, sq)
    st = s.state()
    qoi = json.dumps({"accumulators": [{"name": "shear_p95", "count": 7, "sum": 3.5}]})
    ock.save(s, tmp_path / "o", spec, solid, wall, names=["oxygen"], qoi=qoi)
    lb.checkpoint_write_host(str(tmp_path / "p"), spec, lib_state(st, ["oxygen"], qoi), solid=solid, wall_u=wall)
    for fn in ("manifest.json", ock.RANK_FILE):
        assert same_bytes(tmp_path / "o" / fn, tmp_path / "p" / fn), fn
    m = json.loads((tmp_path / "p" / "manifest.json").read_text())
    assert m["reserved"] == {"particles": False, "rng": False, "stats": True}
    assert m["dtype"] == ("f64" if bits == 64 else "f32") and m["lattice"] == f"D3Q{q}"


@pytest.mark.parametrize("bits", [64, 32])
def test_library_reader_returns_oracle_state(tmp_path, bits):
    s, spec, solid, wall, _ = channel_case(bits)
    st = s.state()
    ock.save(s, tmp_path, spec, solid, wall, names=["oxygen"], qoi='{"a": [1, 2]}', stash="solver")
    r = lb.checkpoint_read_host(str(tmp_path), spec, solid=solid, wall_u=wall)
    assert r["step"] == st["step"] == 9
    assert np.array_equal(r["f"], st["f"]) and np.array_equal(r["moments"], st["moments"])
    assert np.array_equal(r["force_field"], st["force_field"])
    assert r["scalars"][0]["name"] == "oxygen" and r["scalars"][0]["q"] == 7
    assert np.array_equal(r["scalars"][0]["h"], st["scalars"][0]["h"])
    assert np.array_equal(r["scalars"][0]["conc"], st["scalars"][0]["conc"])
    assert r["qoi"] == '{"a": [1, 2]}'


def resume_pair(bits, q, coll, k, m, stash, tmp):
    s, spec, solid, wall, kw = channel_case(bits, q, coll, 7, steps=0)
    cont = o.OracleSolver(s.dims, **kw)
    kc = cont.scalar_enable(0.02, q=7)
    cont.scalar_set(kc, np.where(solid == 0, np.linspace(0.0, 1.0, s.n), 0.0))
    cont.step(k + m)
    s.step(k)
    ock.save(s, tmp, spec, solid, wall, stash=stash)
    fresh = o.OracleSolver(s.dims, **kw)
    fresh.scalar_enable(0.02, q=7)
    ock.restore(fresh, tmp, spec, solid, wall)
    fresh.step(m)
    return cont.state(), fresh.state(), solid


@pytest.mark.parametrize("bits,q,coll", [(32, 19, "trt"), (64, 19, "trt"), (64, 27, "cm")])
def test_oracle_resume_is_bit_exact(tmp_path, bits, q, coll):
    """checkpoint_resume_bit_exact_f32_f64_d2q9_d3q19 (solver.rs:6296-6302):
    run 20 == run 7, save, load, run 13, every array bit for bit."""
    a, b, _ = resume_pair(bits, q, coll, 7, 13, "solver", tmp_path)
    assert a["step"] == b["step"] == 20
    for key in ("f", "ftmp", "moments", "force_field"):
        assert np.array_equal(a[key], b[key]), key
    for x, y in zip(a["scalars"], b["scalars"]):
        for key in ("h", "htmp", "conc"):
            assert np.array_equal(x[key], y[key]), key


def test_zero_stash_resumes_every_fluid_value(tmp_path):
    """With the stash written as zero planes (the library's writer) every
    fluid population, every moment and the scalar still resume bit for bit;
    only never-read solid slots may differ."""
    a, b, solid = resume_pair(64, 19, "trt", 7, 13, "zero", tmp_path)
    fl = solid == 0
    assert np.array_equal(a["f"][:, fl], b["f"][:, fl])
    assert np.array_equal(a["moments"], b["moments"])
    assert np.array_equal(a["scalars"][0]["conc"], b["scalars"][0]["conc"])


def test_stale_stash_and_carried_solid_moments(tmp_path):
    """checkpoint_preserves_stale_stash_and_carried_solid_moments
    (solver.rs:6631-6690)."""
    s, spec, solid, wall, kw = channel_case(32, scalar_q=0, steps=8)
    st = s.state()
    c = int(np.flatnonzero(solid)[0])
    st["moments"][0, c] = 1.2345
    s.set_state(st)
    ock.save(s, tmp_path, spec, solid, wall, stash="solver")
    fresh = o.OracleSolver(s.dims, **kw)
    ock.restore(fresh, tmp_path, spec, solid, wall)
    got = fresh.state()
    assert np.array_equal(got["ftmp"], st["ftmp"].astype(np.float32))
    assert got["moments"][0, c] == np.float32(1.2345)
    r = lb.checkpoint_read_host(str(tmp_path), spec, solid=solid, wall_u=wall)
    assert r["moments"][0, c] == np.float32(1.2345)


def both_fail(path, spec, solid, wall):
    """The oracle's and the library's reader fail with the same code."""
    with pytest.raises(ock.CheckpointError) as eo:
        ock.read(path, spec, solid, wall)
    with pytest.raises(lb.CheckpointError) as el:
        lb.checkpoint_read_host(str(path), spec, solid=solid, wall_u=wall)
    assert el.value.code == eo.value.code, (el.value, eo.value)
    assert el.value.status == lb.ERR_CHECKPOINT
    return el.value


def edit_manifest(path, **changes):
    m = json.loads((path / "manifest.json").read_text())
    for k, v in changes.items():
        m[k] = v
    (path / "manifest.json").write_text(json.dumps(m, indent=2))


def fresh_copy(src, dst):
    if dst.exists():
        shutil.rmtree(dst)
    shutil.copytree(src, dst)
    return dst


def test_mismatch_codes_match_the_reference(tmp_path):
    """checkpoint_layout_and_version_mismatch_are_precise and
    checkpoint_reports_truncated_payload_and_spec_mismatch (solver.rs:
    6366-6421, 6552-6629), plus the other load_into checks."""
    s, spec, solid, wall, _ = channel_case(32, scalar_q=0, steps=3)
    base = tmp_path / "base"
    ock.save(s, base, spec, solid, wall)
    d = tmp_path / "d"

    e = both_fail(fresh_copy(base, d), dict(spec, nu=0.09), solid, wall)
    assert e.code == "CKPT_SCENARIO_MISMATCH" and "scenario_hash differed" in e.message
    assert both_fail(d, dict(spec, periodic=(True, False, False)), solid, wall).code == "CKPT_SCENARIO_MISMATCH"
    assert both_fail(d, dict(spec, force=(2e-6, 0.0, 0.0)), solid, wall).code == "CKPT_SCENARIO_MISMATCH"
    assert both_fail(d, dict(spec, dtype="f64"), solid, wall).code == "CKPT_DTYPE_MISMATCH"
    assert both_fail(d, dict(spec, lattice=27), solid, wall).code == "CKPT_LATTICE_MISMATCH"
    assert both_fail(d, dict(spec, dims=(8, 7, 7)), None, None).code == "CKPT_GEOM_MISMATCH"
    moved = wall.copy().reshape(-1, 3)
    moved[np.flatnonzero(solid)[-1], 0] = 0.02
    assert both_fail(d, spec, solid, moved).code == "CKPT_MASK_MISMATCH"

    edit_manifest(fresh_copy(base, d), format_version=2)
    e = both_fail(d, spec, solid, wall)
    assert e.code == "CKPT_VERSION_MISMATCH" and "format_version 2" in e.message and "migrate" in e.message
    edit_manifest(fresh_copy(base, d), kind="other")
    assert both_fail(d, spec, solid, wall).code == "CKPT_BAD_MAGIC"
    edit_manifest(fresh_copy(base, d), decomp_hash="fnv1a64:0000000000000000")
    e = both_fail(d, spec, solid, wall)
    assert e.code == "CKPT_DECOMP_MISMATCH" and "decomp_hash differed" in e.message
    edit_manifest(fresh_copy(base, d), nranks=2)
    assert both_fail(d, spec, solid, wall).code == "CKPT_RANK_MISMATCH"
    m = json.loads((base / "manifest.json").read_text())
    del m["step"]
    fresh_copy(base, d)
    (d / "manifest.json").write_text(json.dumps(m))
    assert both_fail(d, spec, solid, wall).code == "CKPT_MANIFEST_INVALID"
    (d / "manifest.json").write_text("{ not json")
    assert both_fail(d, spec, solid, wall).code == "CKPT_MANIFEST_INVALID"
    os.remove(d / "manifest.json")
    assert both_fail(d, spec, solid, wall).code == "CKPT_IO"

    rank = ock.RANK_FILE
    clean = (base / rank).read_bytes()
    fresh_copy(base, d)
    bad = bytearray(clean)
    bad[len(bad) // 2] ^= 0x01
    (d / rank).write_bytes(bytes(bad))
    assert both_fail(d, spec, solid, wall).code == "CKPT_PAYLOAD_CORRUPT"
    (d / rank).write_bytes(clean[:-5])
    assert both_fail(d, spec, solid, wall).code in ("CKPT_TRUNCATED", "CKPT_PAYLOAD_CORRUPT")
    (d / rank).write_bytes(clean[:40])
    assert both_fail(d, spec, solid, wall).code == "CKPT_TRUNCATED"
    (d / rank).write_bytes(b"NOTAKPT\x00" + clean[8:])
    assert both_fail(d, spec, solid, wall).code == "CKPT_BAD_MAGIC"


def test_scalar_on_the_hydro_lattice_and_qoi_round_trip(tmp_path):
    """checkpoint_v3_roundtrips_scalar_distribution_state and
    checkpoint_v3_roundtrips_qoi_accumulators_and_manifest_flag (solver.rs:
    6423-6462, 6508-6550) through the library's writer and reader."""
    s, spec, solid, wall, _ = channel_case(64, scalar_q=19, steps=4)
    st = s.state()
    n = s.n
    st["scalars"][0]["h"] = (np.arange(19 * n) * 1e-6).reshape(19, n)
    st["scalars"][0]["conc"] = 0.1 + np.arange(n) * 1e-3
    qoi = json.dumps({"accumulators": [{"name": "shear_p95", "count": 7, "sum": 3.5, "min": 0.1, "max": 1.2,
                                        "reservoir": [0.2, 0.5, 0.9]}]})
    lb.checkpoint_write_host(str(tmp_path), spec, lib_state(st, ["oxygen"], qoi), solid=solid, wall_u=wall)
    m = json.loads((tmp_path / "manifest.json").read_text())
    assert m["reserved"]["stats"] is True and m["reserved"]["particles"] is False and m["reserved"]["rng"] is False
    r = lb.checkpoint_read_host(str(tmp_path), spec, solid=solid, wall_u=wall)
    assert r["scalars"][0]["name"] == "oxygen" and r["scalars"][0]["diffusivity"] == 0.02
    assert np.array_equal(r["scalars"][0]["h"], st["scalars"][0]["h"])
    assert np.array_equal(r["scalars"][0]["conc"], st["scalars"][0]["conc"])
    assert json.loads(r["qoi"]) == json.loads(qoi)
    o_r = ock.read(tmp_path, spec, solid, wall)
    assert np.array_equal(o_r["scalars"][0]["h"], st["scalars"][0]["h"])
    assert not o_r["scalars"][0]["htmp"].any()


def test_padded_masks_follow_the_mask_exchange():
    """Halo rings of the masks: periodic axes wrap (edges and corners
    forwarded), non-periodic faces keep false / zero."""
    dims = (4, 3, 5)
    spec = {"dims": dims, "periodic": (True, False, True), "dtype": "f64"}
    n = 60
    solid = (np.arange(n) % 7 == 0).astype(np.uint8)
    wall = np.arange(3 * n, dtype=np.float64) * 1e-3
    ps, pw = ock.padded_masks(spec, solid, wall)
    ps = ps.reshape(7, 5, 6)
    sg = solid.reshape(5, 3, 4)
    assert np.array_equal(ps[1:-1, 1:-1, 1:-1], sg)
    assert np.array_equal(ps[1:-1, 1:-1, 0], sg[:, :, -1]) and np.array_equal(ps[0, 1:-1, 1:-1], sg[-1])
    assert ps[0, 1:-1, 0].tolist() == sg[-1, :, -1].tolist()
    assert not ps[:, 0, :].any() and not ps[:, -1, :].any()


def test_long_zero_runs_read_back_as_zero(tmp_path):
    """Zero runs of 1 MB and more (the stash planes) are left as file holes;
    the file has the manifest's length, the stash bytes read back as zero
    and the library's reader verifies the payload hash over them."""
    dims = (40, 36, 32)
    n = dims[0] * dims[1] * dims[2]
    spec = dict(dims=dims, lattice=27, collision="cm", dtype="f64", nu=0.02, omega_shear=1.5,
                periodic=(True, True, True), force=(0.0, 0.0, 0.0))
    rng = np.random.default_rng(5)
    st = dict(step=3, f=rng.normal(size=(27, n)), moments=rng.normal(size=(4, n)), force_field=None, scalars=[])
    lb.checkpoint_write_host(str(tmp_path), spec, st)
    m = json.loads((tmp_path / "manifest.json").read_text())
    raw = (tmp_path / ock.RANK_FILE).read_bytes()
    assert len(raw) == m["ranks"][0]["bytes"]
    npad = (dims[0] + 2) * (dims[1] + 2) * (dims[2] + 2)
    head = 40 + 20 * 4  # header + 4 section entries (F, stash, moments, solid)
    stash = raw[head + 27 * npad * 8: head + 2 * 27 * npad * 8]
    assert len(stash) == 27 * npad * 8 > (1 << 20) and not any(stash)
    r = lb.checkpoint_read_host(str(tmp_path), spec)
    assert np.array_equal(r["f"], st["f"]) and np.array_equal(r["moments"], st["moments"])
    assert m["ranks"][0]["payload_hash"] == ock.hash_string(lb.fnv1a64(raw[head:-8]))
