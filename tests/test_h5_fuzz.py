"""Robustness of the native HDF5 reader (include/afid_continua.h) on damaged restart files.

Restart files come from disk, other programs and other machines.  The reader must answer every
damaged file with a status code: no crash, no read outside the file, no negative or overflowing
shape, no unbounded walk of a B-tree whose nodes point back at themselves.  Valid files of the
supported layouts (the version-0 layout the library writes, flat and with nested groups whose
B-trees have two levels, and the version-2 layout of oracle/afid_h5.py) get random byte changes
in their metadata and random truncations; every query must end in AFID_OK, AFID_E_IO or
AFID_E_INVALID.  The mutations run in a
child process, so a crash fails the test instead of ending the test session.
"""
import os
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent(r"""
    import os, sys, tempfile
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "afid-murphfi_b200")); sys.path.insert(0, ROOT)
    import afid_gpu as ag
    from oracle import afid_h5 as h5
    rng = np.random.default_rng(SEED)
    d = tempfile.mkdtemp()
    v0 = os.path.join(d, "v0.h5")
    sets = {f"s{i}": np.arange(i + 1, dtype=np.int32) for i in range(10)}
    sets["var"] = rng.standard_normal((3, 4, 5))
    ag.h5_write(v0, sets)
    v2 = os.path.join(d, "v2.h5")
    h5.write_v2(v2, {"var": rng.standard_normal((3, 4, 5)), "small": np.arange(6, dtype=np.int32)},
                compact=("small",))
    nested = os.path.join(d, "nested.h5")
    tree = {f"big/{k:05d}": np.array([float(k)]) for k in range(300)}
    tree.update({"g/a": np.arange(3, dtype=np.int32), "g/b/c": rng.standard_normal(4), "e": None})
    ag.h5_write(nested, tree)
    names = ["var", "s0", "s9", "small", "big/00007", "big/00299", "g/b/c", "e"]
    statuses = set()
    for base in (v0, v2, nested):
        raw = bytearray(open(base, "rb").read())
        meta = min(len(raw), 16384)
        for trial in range(TRIALS):
            b = bytearray(raw)
            for _ in range(int(rng.integers(1, 6))):
                b[int(rng.integers(0, meta))] = int(rng.integers(0, 256))
            if rng.random() < 0.2:
                b = b[:int(rng.integers(0, len(b)))]
            p = os.path.join(d, "f.h5")
            open(p, "wb").write(b)
            for nm in names:
                try:
                    dt, shape = ag.h5_info(p, nm)
                    assert all(n >= 0 for n in shape), shape
                    if int(np.prod(shape)) <= 1_000_000:
                        ag.h5_read(p, nm)
                    statuses.add(0)
                except ag.AfidError as e:
                    statuses.add(e.status)
    assert statuses <= {0, ag.AFID_E_IO, ag.AFID_E_INVALID}, statuses
    print("statuses", sorted(statuses))
""")


def test_damaged_files_give_status_codes():
    for seed in (1, 2):
        code = f"ROOT = {ROOT!r}\nSEED = {seed}\nTRIALS = 250\n" + CHILD
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
        assert "statuses" in r.stdout


def test_self_referencing_btree_ends(tmp_path):
    """A group B-tree whose root claims five levels and 32 children that all point back at the
    root: the lookup gives up after a bounded number of node visits (AFID_E_IO), in well under
    the time an exhaustive walk (32^5 nodes) would take."""
    import struct
    import time

    import numpy as np

    sys.path.insert(0, ROOT)
    import afid_gpu as ag
    from oracle import afid_h5 as h5
    p = str(tmp_path / "cycle.h5")
    ag.h5_write(p, {f"big/{k:05d}": np.array([1.0]) for k in range(600)})
    f = h5.H5File(p)
    btree = [int.from_bytes(b[:8], "little") for t, _, b in f.messages(f.resolve("big")) if t == 0x11][0]
    raw = bytearray(open(p, "rb").read())
    raw[btree + 5] = 5
    raw[btree + 6:btree + 8] = struct.pack("<H", 32)
    for c in range(32):
        off = btree + 32 + c * 16
        raw[off:off + 8] = struct.pack("<Q", btree)
    open(p, "wb").write(raw)
    t0 = time.perf_counter()
    try:
        ag.h5_read(p, "big/00003")
        status = 0
    except ag.AfidError as e:
        status = e.status
    assert status == ag.AFID_E_IO
    assert time.perf_counter() - t0 < 30.0
