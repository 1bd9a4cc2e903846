"""aw_checkpoint_*: the reference's checkpoint file (include/pic/checkpoint.hpp:
1-17, 31-49) with its array payloads written, and restart. A run restored from
a checkpoint continues bit for bit like the uninterrupted run; the file's
header, manifest and payload follow the reference's layout; bad or foreign
files are refused."""
import struct
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from gpu_helpers import PARTICLE_KEYS, TWO_STREAM, WEIBEL, Setup, n_particles

pytestmark = pytest.mark.gpu

DTYPES = {0: np.float32, 1: np.float64, 2: np.int32, 3: np.uint64}


def parse(path):
    """The reference's layout: header, deck and git blocks, manifest, payloads."""
    b = open(path, "rb").read()
    magic, ver, seed, step, time, sd, eps_l = struct.unpack_from("<IIQqddd", b, 0)
    o = 48
    blocks = []
    for _ in range(2):
        (n,) = struct.unpack_from("<Q", b, o)
        blocks.append(b[o + 8:o + 8 + n].decode())
        o += 8 + n
    (na,) = struct.unpack_from("<I", b, o)
    o += 4
    man = []
    for _ in range(na):
        (nl,) = struct.unpack_from("<I", b, o)
        name = b[o + 4:o + 4 + nl].decode()
        dt, cnt = struct.unpack_from("<IQ", b, o + 4 + nl)
        man.append((name, dt, cnt))
        o += 4 + nl + 12
    arrays = {}
    for name, dt, cnt in man:
        a = np.frombuffer(b, dtype=DTYPES[dt], count=cnt, offset=o)
        arrays[name] = a
        o += a.nbytes
    return dict(magic=magic, version=ver, seed=seed, step=step, time=time, sd=sd, eps_l=eps_l, deck=blocks[0],
                git=blocks[1], manifest=man, arrays=arrays, size=len(b), end=o)


def _make(torch, aw, model):
    if model == "es":
        s = Setup(torch, aw, 64, 64, 64.0, 64.0, n_particles(TWO_STREAM, 64, 64), aw.AW_MODEL_ES, dt=0.1)
        s.ctx.load_species(TWO_STREAM, seed=1, noisy=True)
    else:
        s = Setup(torch, aw, 64, 64, 32.0, 32.0, n_particles(WEIBEL, 64, 64), aw.AW_MODEL_DARWIN, dt=0.05,
                  B0=(0.0, 0.0, 0.2))
        s.ctx.load_species(WEIBEL, seed=1, noisy=True)
    return s


def _state(s):
    return s.parts(), s.ctx.step_diag()


@pytest.mark.parametrize("model", ["es", "darwin"])
@pytest.mark.parametrize("wait", [True, False])
def test_restart_continues_bit_for_bit(torch_cuda, aw, tmp_path, model, wait):
    """Checkpoint at step 30, run to 60 (the Darwin run re-sorts at 50); a fresh
    context restored from the file and run from 30 to 60 ends in the same bits.
    wait=False: the run goes on while the file is written."""
    k1, k2 = 30, 60
    path = tmp_path / "run.ck"
    a = _make(torch_cuda, aw, model)
    b = None
    try:
        a.ctx.init()
        a.ctx.run(0, k1, graph=True)
        a.ctx.checkpoint(path, k1, deck="[grid]\nnx = 64\n", git_hash="abc123", rng_seed=1, wait=wait)
        a.ctx.run(k1, k2 - k1, graph=True)
        a.ctx.checkpoint_wait()
        want_p, want_d = _state(a)
        b = _make(torch_cuda, aw, model)
        for k in PARTICLE_KEYS:                       # the restore overwrites everything
            b.P[k].fill_(0.5)
        info = b.ctx.restore(path)
        assert info["step"] == k1 and info["rng_seed"] == 1
        b.ctx.run(k1, k2 - k1, graph=True)
        got_p, got_d = _state(b)
        for k in want_p:
            assert np.array_equal(got_p[k], want_p[k]), k
        assert got_d == want_d
    finally:
        a.close()
        if b is not None:
            b.close()


def test_file_follows_the_reference_layout(torch_cuda, aw, tmp_path):
    path = tmp_path / "es.ck"
    s = _make(torch_cuda, aw, "es")
    try:
        s.ctx.init()
        s.ctx.run(0, 5, graph=True)
        s.ctx.checkpoint(path, 5, deck="deck text", git_hash="0123abcd", rng_seed=7, sd=2.5, eps_l=0.125)
        p = s.parts()
        f = parse(path)
        assert f["magic"] == 0x57435241 and f["version"] == 1
        assert (f["seed"], f["step"], f["sd"], f["eps_l"]) == (7, 5, 2.5, 0.125)
        assert abs(f["time"] - 0.5) < 1e-12
        assert f["deck"] == "deck text" and f["git"] == "0123abcd"
        names = [m[0] for m in f["manifest"]]
        assert names[:9] == ["x", "y", "ux", "uy", "uz", "w", "cell", "acc_src", "devstate"]
        assert f["end"] == f["size"]                     # payloads follow, nothing else
        for k in PARTICLE_KEYS + ("cell",):
            assert np.array_equal(f["arrays"][k], p[k]), k
        assert np.array_equal(f["arrays"]["Ex"], s.grid("Ex").reshape(-1))
    finally:
        s.close()


def test_bad_files_are_refused(torch_cuda, aw, tmp_path):
    path = tmp_path / "ok.ck"
    s = _make(torch_cuda, aw, "es")
    other = Setup(torch_cuda, aw, 64, 64, 64.0, 64.0, 1000, aw.AW_MODEL_ES, dt=0.1)
    try:
        s.ctx.init()
        s.ctx.checkpoint(path, 0)
        raw = open(path, "rb").read()
        f = parse(path)
        header = f["end"] - sum(a.nbytes for a in f["arrays"].values())
        cases = {"magic": b"XXXX" + raw[4:], "version": raw[:4] + struct.pack("<I", 2) + raw[8:],
                 "schema_only": raw[:header], "truncated": raw[:-16]}
        for name, data in cases.items():
            bad = tmp_path / f"{name}.ck"
            bad.write_bytes(data)
            with pytest.raises(aw.ArcError):
                s.ctx.restore(bad)
        with pytest.raises(aw.ArcError):               # another particle count
            other.ctx.restore(path)
        with pytest.raises(aw.ArcError):
            s.ctx.restore(tmp_path / "missing.ck")
    finally:
        s.close()
        other.close()


def test_reference_reader_reads_the_header(torch_cuda, aw, tmp_path):
    """The reference's own checkpoint_read_header (compiled from its header by the
    shim build) reads what this library writes."""
    exe = ROOT / "arcwarden_b200" / "shim" / "_build" / "ck_manifest"
    if not exe.exists():
        pytest.skip("ck_manifest not built (make -C arcwarden_b200/shim)")
    path = tmp_path / "ref.ck"
    s = _make(torch_cuda, aw, "darwin")
    try:
        s.ctx.init()
        s.ctx.checkpoint(path, 0, deck="d", git_hash="g", rng_seed=3)
        f = parse(path)
        out = subprocess.run([str(exe), str(path)], capture_output=True, text=True, timeout=60)
        assert out.returncode == 0, out.stderr
        lines = out.stdout.split("\n")
        assert lines[0] == "seed 3 step 0 deck d git g"
        for (name, dt, cnt), line in zip(f["manifest"], lines[1:]):
            assert line == f"{name} {dt} {cnt}"
    finally:
        s.close()
