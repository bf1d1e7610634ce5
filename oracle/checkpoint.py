"""Oracle restatement of the reference's v3 checkpoint format (TEST
INFRASTRUCTURE: only tests/ use this module, as the checker of the
library's writer and reader).

Follows crates/lbm-core/src/solver.rs:
  29-44      format version, magic, section ids
  84-118     CheckpointManifest / CheckpointRank / SectionEntry / RankHeader
  831-859    fnv1a64, hash_bytes, hash_u64, hash_f64, hash_real
  881-945    spec_hash (every face closed, no sources, no face patches here)
  947-965    decomp_hash;  967-979 part_mask_hash;  981-1009 names and ids
  1011-1048  push_real_bytes / read_real_bytes
  1108-1198  read_rank_file;  1200-1287 scalar section
  4536-4630  write_part_checkpoint;  4632-4670 manifest;  4715-4724 save
  4759-5060  load_into / load_into_with_layout (checks and their order)
and crates/lbm-core/src/fields.rs:99-150 (halo-padded geometry, halo 1),
halo.rs:457-492 with subdomain.rs:31-44 (mask halos of a monolithic part).

Pinned by: the published FNV-1a 64 test vectors, the reference's own
checkpoint tests (solver.rs:6296-6700: resume bit-exactness, scenario /
version / decomposition mismatch codes, corrupt and truncated payloads,
scalar and QOI round trips, stale stash preservation) restated in
tests/test_oracle_checkpoint.py. No file written by the reference itself is
available (its toolchain is absent), so byte compatibility with
reference-written files rests on this restatement.

The stale stash (ftmp) and the halo rings: the reference writes whatever its
ping-pong partner and halos hold. stash="solver" writes the oracle's own
ftmp (the reference's CpuScalar content); stash="zero" writes zero planes,
the library's choice. Halo cells are written as zero either way.
"""
import json
import os
import struct

import numpy as np

FORMAT_VERSION = 3
MAGIC = b"LBMKPT\x00\x00"
SEC_F_PRIMARY, SEC_STALE_STASH, SEC_MOMENTS, SEC_SOLID, SEC_FORCE_FIELD = 1, 2, 3, 4, 5
SEC_SCALAR_FIELDS, SEC_PHASE_FIELD, SEC_QOI_ACCUMULATORS = 6, 7, 10
RANK_FILE = "rank_0000_part_0000.bin"
FNV_OFFSET, FNV_PRIME, MASK64 = 0xCBF29CE484222325, 0x100000001B3, (1 << 64) - 1
COLLISION_IDS = {"bgk": 1, "trt": 2, "cm": 3}


class CheckpointError(Exception):
    def __init__(self, code, message):
        super().__init__(f"{code}: {message}")
        self.code = code
        self.message = message


def fnv1a64(data, h=FNV_OFFSET):
    for b in bytes(data):
        h = ((h ^ b) * FNV_PRIME) & MASK64
    return h


def hash_string(h):
    return f"fnv1a64:{h:016x}"


def _u64(v):
    return struct.pack("<Q", v)


def _real_bytes(values, f64):
    """push_real_bytes: little-endian f64, or the value rounded to f32."""
    return np.asarray(values, dtype="<f8" if f64 else "<f4").tobytes()


def spec_hash(spec):
    """spec: dims, lattice (19|27), collision ("bgk"|"trt"|"cm"), nu, magic,
    omega_shear, periodic, force, dtype ("f32"|"f64")."""
    f64 = spec["dtype"] == "f64"
    h = FNV_OFFSET
    h = fnv1a64(_u64(3), h)
    h = fnv1a64(_u64(spec["lattice"]), h)
    for d in spec["dims"]:
        h = fnv1a64(_u64(d), h)
    h = fnv1a64(struct.pack("<d", spec["nu"]), h)
    kind = spec["collision"]
    h = fnv1a64(_u64(COLLISION_IDS[kind]), h)
    if kind == "trt":
        h = fnv1a64(struct.pack("<d", spec["magic"]), h)
    elif kind == "cm":
        h = fnv1a64(struct.pack("<d", spec["omega_shear"]), h)
    for p in spec["periodic"]:
        h = fnv1a64(_u64(int(bool(p))), h)
    for _ in range(6):
        h = fnv1a64(_u64(0), h)
    for v in spec["force"]:
        h = fnv1a64(_real_bytes([v], f64), h)
    return h


def decomp_hash(spec):
    h = fnv1a64(_u64(1))
    for p in spec["periodic"]:
        h = fnv1a64(_u64(int(bool(p))), h)
    for v in (0, 0, 0):
        h = fnv1a64(_u64(v), h)
    for d in spec["dims"]:
        h = fnv1a64(_u64(d), h)
    for face in range(6):
        h = fnv1a64(_u64(1 if spec["periodic"][face // 2] else 0), h)
    return h


def padded_shape(dims):
    nx, ny, nz = dims
    return nz + 2, ny + 2, nx + 2


def pad(values, dims, planes):
    """Compact q-major planes -> halo-padded planes, halo zero."""
    nx, ny, nz = dims
    out = np.zeros((planes,) + padded_shape(dims))
    if values is not None:
        out[:, 1:nz + 1, 1:ny + 1, 1:nx + 1] = np.asarray(values, dtype=np.float64).reshape(planes, nz, ny, nx)
    return out.reshape(planes, -1)


def unpad(values, dims, planes):
    nx, ny, nz = dims
    v = np.asarray(values).reshape((planes,) + padded_shape(dims))
    return v[:, 1:nz + 1, 1:ny + 1, 1:nx + 1].reshape(planes, -1)


def padded_masks(spec, solid, wall_u):
    """The masks after the mask exchange of a monolithic part: periodic axes
    wrap, halo cells behind non-periodic faces keep false / zero."""
    nx, ny, nz = spec["dims"]
    n = nx * ny * nz
    solid = np.zeros(n, np.uint8) if solid is None else np.asarray(solid, np.uint8).ravel()
    wall_u = np.zeros((n, 3)) if wall_u is None else np.asarray(wall_u, np.float64).reshape(n, 3)
    ps = np.zeros(padded_shape(spec["dims"]), np.uint8)
    pw = np.zeros(padded_shape(spec["dims"]) + (3,))
    sg, wg = solid.reshape(nz, ny, nx), wall_u.reshape(nz, ny, nx, 3)
    for z in range(-1, nz + 1):
        for y in range(-1, ny + 1):
            for x in range(-1, nx + 1):
                c, ok = [x, y, z], True
                for a, e in enumerate((nx, ny, nz)):
                    if not 0 <= c[a] < e:
                        if not spec["periodic"][a]:
                            ok = False
                        c[a] %= e
                if ok:
                    ps[z + 1, y + 1, x + 1] = 1 if sg[c[2], c[1], c[0]] else 0
                    pw[z + 1, y + 1, x + 1] = wg[c[2], c[1], c[0]]
    return ps.ravel(), pw.reshape(-1, 3)


def mask_hash(spec, solid, wall_u):
    ps, pw = padded_masks(spec, solid, wall_u)
    f64 = spec["dtype"] == "f64"
    h = fnv1a64(_u64(ps.size))
    h = fnv1a64(b"".join(_u64(int(v)) for v in ps), h)
    return fnv1a64(_real_bytes(pw.ravel(), f64), h)


def _manifest(spec, step, nbytes, payload_hash, mhash, stats):
    """serde_json::to_string_pretty of CheckpointManifest (field order of
    the struct, BTreeMap keys sorted)."""
    m = {"kind": "lbmflow-checkpoint", "format_version": FORMAT_VERSION, "step": int(step),
         "time": float(step), "dtype": spec["dtype"], "lattice": f"D3Q{spec['lattice']}",
         "global": list(spec["dims"]), "scenario_hash": hash_string(spec_hash(spec)),
         "decomp_hash": hash_string(decomp_hash(spec)), "nranks": 1,
         "ranks": [{"rank": 0, "part": 0, "file": RANK_FILE, "origin": [0, 0, 0], "core": list(spec["dims"]),
                    "bytes": nbytes, "payload_hash": hash_string(payload_hash), "mask_hash": hash_string(mhash)}],
         "reserved": {"particles": False, "rng": False, "stats": bool(stats)}}
    return json.dumps(m, indent=2)


def write(directory, spec, state, solid=None, wall_u=None, stash="zero"):
    """state: step, f (Q x n), ftmp (for stash="solver"), moments (4 x n),
    force_field (n x 3 | None), scalars [{name, diffusivity, q, h, htmp,
    conc}], qoi (JSON text | None)."""
    f64 = spec["dtype"] == "f64"
    q, dims = spec["lattice"], spec["dims"]
    n = dims[0] * dims[1] * dims[2]
    secs = [(SEC_F_PRIMARY, _real_bytes(pad(state["f"], dims, q), f64)),
            (SEC_STALE_STASH, _real_bytes(pad(state["ftmp"] if stash == "solver" else None, dims, q), f64)),
            (SEC_MOMENTS, _real_bytes(np.asarray(state["moments"]).ravel(), f64))]
    ps, _ = padded_masks(spec, solid, wall_u)
    secs.append((SEC_SOLID, ps.tobytes()))
    if state.get("force_field") is not None:
        secs.append((SEC_FORCE_FIELD, _real_bytes(np.asarray(state["force_field"]).ravel(), f64)))
    if state.get("scalars"):
        b = struct.pack("<I", len(state["scalars"]))
        for x in state["scalars"]:
            name = x["name"].encode()
            sq = int(x["q"])
            npad = pad(None, dims, 1).size
            b += struct.pack("<I", len(name)) + name + struct.pack("<d", x["diffusivity"])
            b += _u64(sq * npad) + _real_bytes(pad(x["h"], dims, sq), f64)
            ht = x.get("htmp") if stash == "solver" else None
            b += _u64(sq * npad) + _real_bytes(pad(ht, dims, sq), f64)
            b += _u64(n) + _real_bytes(np.asarray(x["conc"]).ravel(), f64)
        secs.append((SEC_SCALAR_FIELDS, b))
    if state.get("qoi") is not None:
        secs.append((SEC_QOI_ACCUMULATORS, state["qoi"].encode()))
    payload = b"".join(s for _, s in secs)
    ph = fnv1a64(payload)
    npad = pad(None, dims, 1).size
    head = MAGIC + struct.pack("<IBBHHH", FORMAT_VERSION, 0, 1 if f64 else 0, 300 + q, q, 3)
    head += _u64(npad) + _u64(n) + struct.pack("<I", len(secs))
    off = 0
    for sid, s in secs:
        head += struct.pack("<IQQ", sid, off, len(s))
        off += len(s)
    blob = head + payload + _u64(ph)
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, RANK_FILE), "wb") as fh:
        fh.write(blob)
    with open(os.path.join(directory, "manifest.json"), "w") as fh:
        fh.write(_manifest(spec, state["step"], len(blob), ph, mask_hash(spec, solid, wall_u),
                           state.get("qoi") is not None))


def _reals(b, expected, f64):
    w = 8 if f64 else 4
    if len(b) != expected * w:
        raise CheckpointError("CKPT_GEOM_MISMATCH", f"section length {len(b)} does not match expected {expected} "
                                                    f"values of {w} bytes")
    return np.frombuffer(b, dtype="<f8" if f64 else "<f4").astype(np.float64)


class _Cursor:
    def __init__(self, b):
        self.b, self.pos = b, 0

    def take(self, k):
        if len(self.b) - self.pos < k:
            raise CheckpointError("CKPT_TRUNCATED", "rank file ended before the declared header/table/payload")
        out = self.b[self.pos:self.pos + k]
        self.pos += k
        return out

    def unpack(self, fmt):
        return struct.unpack("<" + fmt, self.take(struct.calcsize("<" + fmt)))


def read(directory, spec, solid=None, wall_u=None):
    """load_into's checks in the reference's order; returns the state dict
    (f, ftmp, moments, force_field, scalars with h/htmp/conc, qoi, step)."""
    f64 = spec["dtype"] == "f64"
    q, dims = spec["lattice"], spec["dims"]
    n = dims[0] * dims[1] * dims[2]
    npad = pad(None, dims, 1).size
    try:
        with open(os.path.join(directory, "manifest.json")) as fh:
            text = fh.read()
    except OSError as e:
        raise CheckpointError("CKPT_IO", str(e)) from None
    try:
        m = json.loads(text)
        fields = ("kind", "format_version", "step", "time", "dtype", "lattice", "global", "scenario_hash",
                  "decomp_hash", "nranks", "ranks", "reserved")
        missing = [k for k in fields if k not in m]
        if missing:
            raise ValueError(f"missing field `{missing[0]}`")
    except ValueError as e:
        raise CheckpointError("CKPT_MANIFEST_INVALID", str(e)) from None
    if m["kind"] != "lbmflow-checkpoint":
        raise CheckpointError("CKPT_BAD_MAGIC", f"manifest kind is {m['kind']}")
    if m["format_version"] != FORMAT_VERSION:
        raise CheckpointError("CKPT_VERSION_MISMATCH",
                              f"checkpoint format_version {m['format_version']} differs from supported "
                              f"{FORMAT_VERSION}; rerun from the original scenario or migrate with a checkpoint "
                              "upgrader before restart")
    if m["dtype"] != spec["dtype"]:
        raise CheckpointError("CKPT_DTYPE_MISMATCH", f"checkpoint dtype {m['dtype']} differs from run dtype "
                                                     f"{spec['dtype']}")
    if m["lattice"] != f"D3Q{q}":
        raise CheckpointError("CKPT_LATTICE_MISMATCH", f"checkpoint lattice {m['lattice']} differs from run "
                                                       f"lattice D3Q{q}")
    if list(m["global"]) != list(dims):
        raise CheckpointError("CKPT_GEOM_MISMATCH", f"checkpoint global {m['global']} differs from run "
                                                    f"{list(dims)}")
    cur = hash_string(spec_hash(spec))
    if m["scenario_hash"] != cur:
        raise CheckpointError("CKPT_SCENARIO_MISMATCH",
                              f"scenario_hash differed: checkpoint={m['scenario_hash']} current={cur}")
    cur = hash_string(decomp_hash(spec))
    if m["decomp_hash"] != cur:
        raise CheckpointError("CKPT_DECOMP_MISMATCH",
                              f"decomp_hash differed: checkpoint={m['decomp_hash']} current={cur}")
    if m["nranks"] != 1:
        raise CheckpointError("CKPT_RANK_MISMATCH", f"checkpoint rank count {m['nranks']} differs from current 1")
    mine = [e for e in m["ranks"] if e["rank"] == 0]
    if len(mine) != 1:
        raise CheckpointError("CKPT_DECOMP_MISMATCH", f"checkpoint has {len(mine)} payload parts for rank 0, "
                                                      "current owner has 1")
    e = mine[0]
    if list(e["origin"]) != [0, 0, 0] or list(e["core"]) != list(dims):
        raise CheckpointError("CKPT_GEOM_MISMATCH", "part geometry differed")
    cur = hash_string(mask_hash(spec, solid, wall_u))
    if e["mask_hash"] != cur:
        raise CheckpointError("CKPT_MASK_MISMATCH", f"mask_hash differed for rank=0 part={e['part']}: "
                                                    f"checkpoint={e['mask_hash']} current={cur}")
    try:
        with open(os.path.join(directory, e["file"]), "rb") as fh:
            blob = fh.read()
    except OSError as err:
        raise CheckpointError("CKPT_IO", str(err)) from None
    c = _Cursor(blob)
    if c.take(8) != MAGIC:
        raise CheckpointError("CKPT_BAD_MAGIC", "rank file magic is not LBMKPT")
    (ver,) = c.unpack("I")
    if ver != FORMAT_VERSION:
        raise CheckpointError("CKPT_VERSION_MISMATCH", f"rank file format_version {ver} differs from supported "
                                                       f"{FORMAT_VERSION}")
    endian, dtype, lat, hq, hd, hnp, hnc, count = c.unpack("BBHHHQQI")
    if endian != 0:
        raise CheckpointError("CKPT_BAD_MAGIC", "cross-endian checkpoints are not supported")
    table = [c.unpack("IQQ") for _ in range(count)]
    if len(blob) - c.pos < 8:
        raise CheckpointError("CKPT_TRUNCATED", "rank file is missing payload hash trailer")
    payload = blob[c.pos:len(blob) - 8]
    (ph,) = struct.unpack("<Q", blob[-8:])
    if fnv1a64(payload) != ph:
        raise CheckpointError("CKPT_PAYLOAD_CORRUPT", "rank file payload hash does not match its contents")
    secs = {}
    for sid, off, ln in table:
        if off + ln > len(payload):
            raise CheckpointError("CKPT_TRUNCATED", f"section {sid} range {off}..{off + ln} exceeds payload "
                                                    f"length {len(payload)}")
        secs[sid] = payload[off:off + ln]
    if dtype != (1 if f64 else 0):
        raise CheckpointError("CKPT_DTYPE_MISMATCH", "rank file dtype differs from requested run precision")
    if lat != 300 + q or hq != q or hd != 3:
        raise CheckpointError("CKPT_LATTICE_MISMATCH", "rank file lattice metadata differs from requested lattice")
    if hnp != npad or hnc != n:
        raise CheckpointError("CKPT_GEOM_MISMATCH", f"rank file np/n_core {hnp}/{hnc} differs from current "
                                                    f"{npad}/{n}")
    if hash_string(ph) != e["payload_hash"]:
        raise CheckpointError("CKPT_PAYLOAD_CORRUPT", "rank payload hash differs from manifest")

    def required(sid, name):
        if sid not in secs:
            raise CheckpointError("CKPT_TRUNCATED", f"checkpoint is missing required section {name}")
        return secs[sid]
    st = {"step": m["step"]}
    st["f"] = unpad(_reals(required(SEC_F_PRIMARY, "F_PRIMARY"), q * npad, f64), dims, q)
    st["ftmp"] = unpad(_reals(required(SEC_STALE_STASH, "STALE_STASH"), q * npad, f64), dims, q)
    st["moments"] = _reals(required(SEC_MOMENTS, "MOMENTS"), 4 * n, f64).reshape(4, n)
    if SEC_SOLID in secs:
        if len(secs[SEC_SOLID]) != npad:
            raise CheckpointError("CKPT_GEOM_MISMATCH", "solid section length differs from current padded geometry")
        ps, _ = padded_masks(spec, solid, wall_u)
        if not np.array_equal(np.frombuffer(secs[SEC_SOLID], np.uint8) != 0, ps != 0):
            raise CheckpointError("CKPT_MASK_MISMATCH", "serialized solid mask differs from rebuilt mask")
    st["force_field"] = (_reals(secs[SEC_FORCE_FIELD], 3 * n, f64).reshape(n, 3)
                         if SEC_FORCE_FIELD in secs else None)
    st["scalars"] = []
    if SEC_SCALAR_FIELDS in secs:
        sc = _Cursor(secs[SEC_SCALAR_FIELDS])
        w = 8 if f64 else 4
        (k,) = sc.unpack("I")
        for _ in range(k):
            (nl,) = sc.unpack("I")
            name = sc.take(nl).decode()
            (d,) = sc.unpack("d")
            (hl,) = sc.unpack("Q")
            hb = sc.take(hl * w)
            (tl,) = sc.unpack("Q")
            tb = sc.take(tl * w)
            (cl,) = sc.unpack("Q")
            cb = sc.take(cl * w)
            sq = hl // npad
            if hl % npad or sq not in (7, q) or tl != hl or cl != n:
                raise CheckpointError("CKPT_GEOM_MISMATCH", "scalar checkpoint section length differs from "
                                                            "current geometry")
            st["scalars"].append({"name": name, "diffusivity": d, "q": sq,
                                  "h": unpad(_reals(hb, hl, f64), dims, sq),
                                  "htmp": unpad(_reals(tb, tl, f64), dims, sq),
                                  "conc": _reals(cb, cl, f64)})
        if sc.pos != len(sc.b):
            raise CheckpointError("CKPT_PAYLOAD_CORRUPT", "scalar checkpoint section has trailing bytes")
    st["qoi"] = secs[SEC_QOI_ACCUMULATORS].decode() if SEC_QOI_ACCUMULATORS in secs else None
    if st["qoi"] is not None:
        json.loads(st["qoi"])
    return st


def solver_spec(s, collision, nu, magic, omega_shear, periodic, force):
    """spec dict of an OracleSolver built with these parameters."""
    return {"dims": tuple(s.dims), "lattice": s.q, "collision": collision, "nu": nu, "magic": magic,
            "omega_shear": omega_shear, "periodic": tuple(bool(p) for p in periodic), "force": tuple(force),
            "dtype": "f64" if s.real_bits == 64 else "f32"}


def save(solver, directory, spec, solid=None, wall_u=None, names=None, qoi=None, stash="zero"):
    """Solver::save of an OracleSolver."""
    st = solver.state()
    for k, x in enumerate(st["scalars"]):
        x["name"] = names[k] if names else f"scalar{k}"
    st["qoi"] = qoi
    write(directory, spec, st, solid, wall_u, stash=stash)


def restore(solver, directory, spec, solid=None, wall_u=None):
    """Solver::restore of an OracleSolver (its scalars must be enabled)."""
    st = read(directory, spec, solid, wall_u)
    solver.set_state(st)
    return st
