"""Host side of the case layer (include/orchard_b200_cases.h), no GPU needed.

Config files, describe(), the case geometry and the SLVCHKP1 checkpoint codec
against the reference's own code (oracle/_ref, compiled in place from the
reference sources) and against the committed fixtures it wrote
(tests/golden/cases/, made by tests/golden/make_case_golden.py).  The
expectations follow the reference's checkpoint tests
(tests/test_runtime.cpp:2014-2190): bitwise round trip, checksum, version,
build-hash and configuration checks.
"""
import json
import math
import os
import struct
import sys

import numpy as np
import pytest

import solver_b200.cases as cs

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "cases")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import pyoracle as po  # noqa: E402


@pytest.fixture(scope="module")
def refio():
    if not os.path.exists(po.REF_SO):
        pytest.skip("reference build (oracle/_ref) not present")
    return po.ReferenceIO()


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


TG_TEXTS = {
    "tg_3d": "nx = 24\nny = 16\nnz = 8\nviscosity = 0.000625\ncfl_limit = 0.5\nfinal_time = 0.0123\n"
             "poisson_max_iterations = 400\npoisson_tolerance = 1e-12\nvalidate_energy = off\n",
    "tg_comments": "# header\n\n  nx=64   # inline\nny = 64\n\tviscosity = 1e-3 \nbackend = cpu\n",
    "tg_defaults": "",
}

CAVITY_TEXTS = {
    "cavity_1024": "nx = 1024\nny = 1024\nreynolds = 100\nlid_velocity = 1.0\ncfl_limit = 0.5\n"
                   "max_steps = 200000\nmin_steps = 400\nsteady_tolerance = 1e-8\n"
                   "poisson_max_iterations = 400\npoisson_tolerance = 1e-12\nvalidate_reference = yes\n",
    "cavity_odd": "nx = 48\nny = 40\nreynolds = 400\nlid_velocity = 2\nsteady_tolerance = 3.5e-9\n"
                  "validate_reference = 0\n",
}


@pytest.mark.parametrize("name", sorted(TG_TEXTS))
def test_taylor_green_config_matches_reference(tmp_path, refio, name):
    path = _write(tmp_path, name + ".cfg", TG_TEXTS[name])
    ours = cs.load_taylor_green_config(path)
    theirs, validate, text = refio.tg_config_load(path)
    for key in ("nx", "ny", "nz", "viscosity", "cfl_limit", "final_time", "poisson_max_iterations",
                "poisson_tolerance"):
        assert getattr(ours, key) == getattr(theirs, key), key
    assert ours.validate_energy == validate
    assert cs.describe(ours) == text
    # geometry and step count of the case
    grid, bc, dt, steps = cs.taylor_green_case(ours)
    rg = refio.tg_grid(theirs)
    assert (grid.nx, grid.ny, grid.nz, grid.dx, grid.dy, grid.dz) == (rg.nx, rg.ny, rg.nz, rg.dx, rg.dy, rg.dz)
    assert dt == refio.tg_dt(theirs)
    assert steps == math.ceil(ours.final_time / dt)
    rbc = refio.tg_bc(theirs)
    assert [bc.faces[f].type for f in range(6)] == [rbc.faces[f].type for f in range(6)]


@pytest.mark.parametrize("name", sorted(CAVITY_TEXTS))
def test_cavity_config_matches_reference(tmp_path, refio, name):
    path = _write(tmp_path, name + ".cfg", CAVITY_TEXTS[name])
    ours = cs.load_lid_driven_cavity_config(path)
    theirs, validate, text = refio.cavity_config_load(path)
    for key in ("nx", "ny", "reynolds", "lid_velocity", "cfl_limit", "max_steps", "min_steps",
                "steady_tolerance", "poisson_max_iterations", "poisson_tolerance"):
        assert getattr(ours, key) == getattr(theirs, key), key
    assert ours.validate_reference == validate
    assert cs.describe(ours) == text
    grid, bc, nu, dt = cs.lid_driven_cavity_case(ours)
    rg = refio.cavity_grid(theirs)
    assert (grid.nx, grid.ny, grid.nz, grid.dx, grid.dy, grid.dz) == (rg.nx, rg.ny, rg.nz, rg.dx, rg.dy, rg.dz)
    assert dt == refio.cavity_dt(theirs)
    assert nu == ours.lid_velocity / ours.reynolds
    rbc = refio.cavity_bc(theirs)
    for f in range(6):
        assert bc.faces[f].type == rbc.faces[f].type
        assert list(bc.faces[f].velocity) == list(rbc.faces[f].velocity)


BAD_TG = [
    ("nx = 8\nfoo = 1\n", "unsupported Taylor-Green config key: foo"),
    ("nx = 8\njust words\n", "invalid config line 2: just words"),
    ("validate_energy = maybe\n", "invalid boolean value: maybe"),
    ("backend = gpu\n", "invalid Taylor-Green backend value: gpu"),
    ("nz = 0\n", "Taylor-Green config expects positive nx, ny, and nz"),
    ("viscosity = -1\n", "Taylor-Green config expects viscosity > 0"),
    ("final_time = 0\n", "Taylor-Green config expects final_time > 0"),
    ("poisson_tolerance = 0\n", "Taylor-Green config expects positive Poisson controls"),
]

BAD_CAVITY = [
    ("nx = 8\nbar = 2\n", "unsupported cavity config key: bar"),
    ("reynolds = 0\n", "lid-driven cavity config expects reynolds > 0"),
    ("min_steps = -1\n", "lid-driven cavity config expects non-negative step controls"),
    ("lid_velocity = 0\n", "lid-driven cavity config expects lid_velocity > 0"),
]


@pytest.mark.parametrize("text,message", BAD_TG)
def test_taylor_green_config_errors_match_reference(tmp_path, refio, text, message):
    path = _write(tmp_path, "bad.cfg", text)
    with pytest.raises(Exception) as ours:
        cs.load_taylor_green_config(path)
    with pytest.raises(Exception) as theirs:
        refio.tg_config_load(path)
    assert str(ours.value) == str(theirs.value) == message


@pytest.mark.parametrize("text,message", BAD_CAVITY)
def test_cavity_config_errors_match_reference(tmp_path, refio, text, message):
    path = _write(tmp_path, "bad.cfg", text)
    with pytest.raises(Exception) as ours:
        cs.load_lid_driven_cavity_config(path)
    with pytest.raises(Exception) as theirs:
        refio.cavity_config_load(path)
    assert str(ours.value) == str(theirs.value) == message


def test_missing_config_file_message(tmp_path):
    with pytest.raises(RuntimeError, match="unable to open Taylor-Green config: "):
        cs.load_taylor_green_config(str(tmp_path / "none.cfg"))
    with pytest.raises(RuntimeError, match="unable to open cavity config: "):
        cs.load_lid_driven_cavity_config(str(tmp_path / "none.cfg"))


def test_fnv_and_build_hash():
    # FNV-1a 64 of "" and "a" (published test values of the hash)
    assert cs.fnv1a64(b"") == 0xcbf29ce484222325
    assert cs.fnv1a64(b"a") == 0xaf63dc4c8601ec8c
    h = cs.build_hash("Orchard Flow", "0.1.0", "GNU", "13.3.0", "deterministic", False)
    assert h == cs.fnv1a64(b"Orchard Flow|0.1.0|GNU|13.3.0|deterministic|strict")
    assert cs.library_build_hash() not in (0, h)


# ---- SLVCHKP1 against the reference's own writer ------------------------------------

def _golden():
    with open(os.path.join(GOLD, "cavity_24.json")) as f:
        info = json.load(f)
    arrs = np.load(os.path.join(GOLD, "cavity_24.npz"))
    cfg = cs.LidDrivenCavityConfig(**{k: info["config"][k] for k in
                                      ("nx", "ny", "reynolds", "lid_velocity", "cfl_limit", "max_steps",
                                       "min_steps", "steady_tolerance", "poisson_max_iterations",
                                       "poisson_tolerance")},
                                   validate_reference=info["validate_reference"])
    state = {k: arrs[k] for k in ("u", "v", "w", "adv_u", "adv_v", "adv_w", "p")}
    state["has_previous_advection"] = int(arrs["has_prev"])
    state["metrics"] = dict(info["metrics"])
    return cfg, state, info


def _ref_hash(info):
    parts = info["build_description"].split("|")
    return cs.build_hash(*parts[:5], fast_math=parts[5] == "fast-math")


def test_reference_build_hash_is_the_fnv_of_its_build_description():
    cfg, state, info = _golden()
    assert _ref_hash(info) == int(info["build_hash"])
    assert cs.fnv1a64(cs.describe(cfg).encode()) == int(info["configuration_hash"])


def test_checkpoint_bytes_equal_reference_writer(tmp_path):
    cfg, state, info = _golden()
    path = str(tmp_path / "ours.chk")
    cs.write_cavity_checkpoint_host(path, cfg, state, build_hash=_ref_hash(info))
    with open(path, "rb") as f, open(os.path.join(GOLD, "cavity_24.chk"), "rb") as g:
        assert f.read() == g.read()


def test_checkpoint_load_of_reference_file_is_bitwise(tmp_path):
    cfg, state, info = _golden()
    loaded, meta = cs.load_cavity_checkpoint_host(os.path.join(GOLD, "cavity_24.chk"), cfg,
                                                  build_hash=_ref_hash(info))
    for k in ("u", "v", "w", "adv_u", "adv_v", "adv_w", "p"):
        assert np.array_equal(loaded[k].view(np.uint64), state[k].view(np.uint64)), k
    assert loaded["has_previous_advection"] == state["has_previous_advection"]
    for k, v in state["metrics"].items():
        if k != "max_divergence_l2":
            assert loaded["metrics"][k] == v, k
    assert meta["format_version"] == 1 and meta["scalar_bytes"] == 8
    assert meta["checksum"] == int(info["checksum"])
    assert meta["build_hash"] == int(info["build_hash"])
    assert meta["configuration_hash"] == int(info["configuration_hash"])


def test_reference_loads_our_checkpoint(tmp_path, refio):
    cfg, state, info = _golden()
    path = str(tmp_path / "ours.chk")
    cs.write_cavity_checkpoint_host(path, cfg, state, build_hash=_ref_hash(info))
    cc = po.cavity_config(cfg.nx, cfg.ny, cfg.reynolds, cfg.lid_velocity, cfg.cfl_limit, cfg.max_steps,
                          cfg.min_steps, cfg.steady_tolerance, cfg.poisson_max_iterations,
                          cfg.poisson_tolerance)
    s, meta = refio.cavity_checkpoint_load(path, cc, cfg.validate_reference)
    for k in ("u", "v", "w", "adv_u", "adv_v", "adv_w", "p"):
        assert np.array_equal(getattr(s, k), state[k]), k


def _corrupt(src, dst, fn):
    with open(src, "rb") as f:
        b = bytearray(f.read())
    fn(b)
    with open(dst, "wb") as f:
        f.write(bytes(b))
    return dst


def _refresh_checksum(b):
    payload = bytes(b[28:])
    b[12:20] = struct.pack("<Q", len(payload))
    b[20:28] = struct.pack("<Q", cs.fnv1a64(payload))


def _section(b, tag):
    at = 28
    while at < len(b):
        n = struct.unpack_from("<Q", b, at + 4)[0]
        if bytes(b[at:at + 4]) == tag:
            return at + 12, n
        at += 12 + n
    raise KeyError(tag)


CORRUPTIONS = {
    "checksum": (lambda b: b.__setitem__(len(b) - 3, b[len(b) - 3] ^ 0xFF),
                 "checkpoint checksum verification failed"),
    "version": (lambda b: b.__setitem__(slice(8, 12), struct.pack("<I", 2)),
                "unsupported checkpoint format version: 2"),
    "magic": (lambda b: b.__setitem__(0, ord("X")), "checkpoint magic mismatch: "),
    "length": (lambda b: b.extend(b"\0"), "checkpoint payload length does not match the file size"),
    "too_small": (lambda b: b.__delitem__(slice(20, None)), "checkpoint file is too small: "),
    "precision": (lambda b: (b.__setitem__(slice(_section(b, b"META")[0], _section(b, b"META")[0] + 4),
                                           struct.pack("<I", 4)), _refresh_checksum(b)),
                  "checkpoint precision does not match the current solver precision"),
    "config_hash": (lambda b: (b.__setitem__(slice(_section(b, b"META")[0] + 12, _section(b, b"META")[0] + 20),
                                             struct.pack("<Q", 12345)), _refresh_checksum(b)),
                    "checkpoint configuration hash does not match the requested config"),
    "missing_section": (lambda b: (b.__setitem__(slice(_section(b, b"PRST")[0] - 12, _section(b, b"PRST")[0] - 8),
                                                 b"XXXX"), _refresh_checksum(b)),
                        "checkpoint is missing one or more required sections"),
    "field_extent": (lambda b: (b.__setitem__(slice(_section(b, b"VELX")[0], _section(b, b"VELX")[0] + 4),
                                              struct.pack("<I", 7)), _refresh_checksum(b)),
                     "checkpoint field extent does not match the current layout"),
}


@pytest.mark.parametrize("kind", sorted(CORRUPTIONS))
def test_checkpoint_rejections_match_reference(tmp_path, refio, kind):
    cfg, state, info = _golden()
    fn, message = CORRUPTIONS[kind]
    path = _corrupt(os.path.join(GOLD, "cavity_24.chk"), str(tmp_path / "bad.chk"), fn)
    with pytest.raises(RuntimeError) as ours:
        cs.load_cavity_checkpoint_host(path, cfg, build_hash=_ref_hash(info))
    cc = po.cavity_config(cfg.nx, cfg.ny, cfg.reynolds, cfg.lid_velocity, cfg.cfl_limit, cfg.max_steps,
                          cfg.min_steps, cfg.steady_tolerance, cfg.poisson_max_iterations,
                          cfg.poisson_tolerance)
    with pytest.raises(Exception) as theirs:
        refio.cavity_checkpoint_load(path, cc, cfg.validate_reference)
    assert str(ours.value) == str(theirs.value)
    assert str(ours.value).startswith(message)


def test_checkpoint_rejects_other_build_and_config():
    cfg, state, info = _golden()
    path = os.path.join(GOLD, "cavity_24.chk")
    with pytest.raises(RuntimeError, match="checkpoint build hash does not match the current executable"):
        cs.load_cavity_checkpoint_host(path, cfg)  # this library's own build hash
    other = cs.LidDrivenCavityConfig(**{**cfg.__dict__, "steady_tolerance": 2e-7})
    with pytest.raises(RuntimeError, match="checkpoint configuration hash does not match the requested config"):
        cs.load_cavity_checkpoint_host(path, other, build_hash=_ref_hash(info))


def test_checkpoint_round_trip_with_library_hash(tmp_path):
    cfg, state, info = _golden()
    path = str(tmp_path / "own.chk")
    cs.write_cavity_checkpoint_host(path, cfg, state)
    loaded, meta = cs.load_cavity_checkpoint_host(path, cfg)
    assert meta["build_hash"] == cs.library_build_hash()
    for k in ("u", "v", "w", "adv_u", "adv_v", "adv_w", "p"):
        assert np.array_equal(loaded[k], state[k])


CONFIGS = os.path.join(os.path.dirname(HERE), "solver_b200", "configs")


@pytest.mark.parametrize("name,steps", [("taylor_green_2d_128.cfg", 100), ("taylor_green_3d_256.cfg", 200)])
def test_shipped_taylor_green_configs(refio, name, steps):
    path = os.path.join(CONFIGS, name)
    ours = cs.load_taylor_green_config(path)
    _, _, text = refio.tg_config_load(path)
    assert cs.describe(ours) == text
    assert cs.taylor_green_case(ours)[3] == steps


@pytest.mark.parametrize("name", ["lid_driven_cavity_re100_128.cfg", "lid_driven_cavity_re100_1024.cfg"])
def test_shipped_cavity_configs(refio, name):
    path = os.path.join(CONFIGS, name)
    ours = cs.load_lid_driven_cavity_config(path)
    _, _, text = refio.cavity_config_load(path)
    assert cs.describe(ours) == text
    assert ours.steady_tolerance == 1e-8 and ours.reynolds == 100.0


BIN = os.path.join(os.path.dirname(HERE), "solver_b200", "bin")

CLI_CASES = [
    ("solver_cavity", ["--foo"]),
    ("solver_cavity", ["/nonexistent/cavity.cfg"]),
    ("solver_cavity", ["--steps"]),
    ("solver_cavity", ["a.cfg", "b.cfg"]),
    ("solver_taylor_green", ["--vtk-out"]),
    ("solver_taylor_green", ["--bogus", "x"]),
    ("solver_taylor_green", ["/nonexistent/tg.cfg"]),
]


@pytest.mark.parametrize("tool,args", CLI_CASES)
def test_cli_argument_errors_match_reference(tool, args):
    """Argument and config errors of the CLIs come before any device work, so
    they are compared with the reference's CLIs on the CPU: same stderr line,
    same exit status."""
    import subprocess
    ref = os.path.join(os.path.dirname(po.REF_SO), tool)
    ours = os.path.join(BIN, tool)
    if not os.path.exists(ref):
        pytest.skip("reference CLIs (oracle/_ref) not built")
    a = subprocess.run([ours, *args], capture_output=True, text=True, timeout=60)
    b = subprocess.run([ref, *args], capture_output=True, text=True, timeout=60)
    assert a.returncode == b.returncode == 1
    assert a.stderr == b.stderr
    assert a.stdout == b.stdout == ""
