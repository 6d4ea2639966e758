"""Dense and batched filter + group-by against the oracle, byte for byte.

The single-table FILTER -> SELECT ... GROUP BY shape takes the dense group-by (one
persistent launch; stats.plan == 1); the same scripts on a plain session take the operator
path. A batch of scripts (alk_session_execute_batch) runs every dense group-by in one
launch and must give each script's own result; scripts of other shapes and failing
scripts in the batch keep their one-at-a-time behaviour."""
import os

import pytest

import alenka_b200 as ab
from alenka_b200 import workloads as wl

from . import _oracle
from .test_gpu_parity import _read, _run_both_or_error

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def flats(tmp_path_factory):
    out = []
    for i, (rows, seg, delta) in enumerate([(300_000, 100_000, False), (250_000, 0, False),
                                            (200_000, 70_000, True)]):
        d = tmp_path_factory.mktemp(f"flat{i}")
        ab.gen_lineitem_flat(str(d), rows, seg, 31 + i, delta=delta)
        out.append(str(d))
    return out


def _flat(filt, select, out="g.txt", group="l_returnflag, l_linestatus"):
    return (f"LF := FILTER lineitem BY {filt};\n"
            f"R := SELECT {select} FROM LF GROUP BY {group};\n"
            f"STORE R INTO '{out}' USING ('|');\n")


SHAPES = {
    "q1": None,  # the config-1 script itself
    "minmax_avg": _flat("l_shipdate < 19960101",
                        "l_returnflag AS f, l_linestatus AS s, MIN(l_quantity) AS mn, MAX(l_extendedprice) AS mx, "
                        "AVG(l_quantity) AS aq, COUNT(l_orderkey) AS c"),
    "range_one_key": _flat("l_shipdate >= 19940101 AND l_shipdate < 19950101",
                           "l_returnflag AS f, SUM(l_extendedprice*(1-l_discount)) AS rev, COUNT(l_orderkey) AS c",
                           group="l_returnflag"),
    "decimal_const": _flat("l_discount >= 0.05 AND l_quantity < 24",
                           "l_linestatus AS s, SUM(l_extendedprice*l_discount) AS rev, SUM(l_quantity) AS q, "
                           "COUNT(l_orderkey) AS c", group="l_linestatus"),
    "empty": _flat("l_shipdate < 19000101", "l_returnflag AS f, SUM(l_quantity) AS q, COUNT(l_orderkey) AS c",
                   group="l_returnflag"),
    "all_rows": _flat("l_shipdate > 19000101", "l_returnflag AS f, l_linestatus AS s, SUM(l_quantity) AS q, "
                      "SUM(2*l_extendedprice-l_extendedprice) AS p, COUNT(l_orderkey) AS c"),
}


@pytest.mark.parametrize("which", [0, 1, 2])
@pytest.mark.parametrize("shape", sorted(SHAPES))
def test_dense_groupby_matches_oracle(flats, which, shape):
    d = flats[which]
    script = SHAPES[shape] or wl.flat_script(7, out="g.txt")
    o, g = _run_both_or_error(d, script, "g.txt")
    assert o == g
    if o is not None and shape != "empty":
        with ab.Session(d) as s:
            s.execute(script)
            assert s.stats().plan == 1  # the dense group-by ran


def test_batch_equals_one_at_a_time(flats, tmp_path):
    scripts, dirs = [], []
    k = 0
    for which, d in enumerate(flats):
        for seed in range(6):
            scripts.append((d, wl.flat_script(100 + seed, out=f"b{k}.txt"), f"b{k}.txt"))
            k += 1
        for name in ("minmax_avg", "range_one_key"):
            scripts.append((d, SHAPES[name].replace("g.txt", f"b{k}.txt"), f"b{k}.txt"))
            k += 1
    # the scripts of one session must share its data directory: one batch per directory
    for d in flats:
        mine = [(sc, o) for dd, sc, o in scripts if dd == d]
        want = []
        for sc, o in mine:
            _oracle.execute(d, sc.replace(o, "oracle_" + o))
            want.append(_read(os.path.join(d, "oracle_" + o)))
        with ab.Session(d) as s:
            s.execute_batch([sc for sc, _ in mine])
            st = s.stats()
            assert st.plan == 1
        for (sc, o), w in zip(mine, want):
            assert _read(os.path.join(d, o)) == w, o


def test_batch_isolates_failures_and_other_shapes(flats):
    d = flats[0]
    good = wl.flat_script(3, out="i0.txt")
    bad = "LF := FILTER lineitem BY l_shipdate < 19960101;\nR := SELECT nosuch AS x, COUNT(l_orderkey) AS c " \
          "FROM LF GROUP BY nosuch;\nSTORE R INTO 'i1.txt' USING ('|');\n"
    plain_shape = ("LF := FILTER lineitem BY l_shipdate < 19960101;\n"
                   "R := SELECT l_orderkey AS k, COUNT(l_orderkey) AS c FROM LF GROUP BY l_orderkey;\n"
                   "STORE R INTO 'i2.txt' USING ('|');\n")  # key domain too wide: operator path
    good2 = wl.flat_script(4, out="i3.txt")
    want = {}
    for sc, o in ((good, "i0.txt"), (plain_shape, "i2.txt"), (good2, "i3.txt")):
        _oracle.execute(d, sc.replace(o, "oracle_" + o))
        want[o] = _read(os.path.join(d, "oracle_" + o))
    with ab.Session(d) as s:
        with pytest.raises(ab.AlenkaError) as e:
            s.execute_batch([good, bad, plain_shape, good2])
        assert "script 1" in str(e.value)
    for o, w in want.items():
        assert _read(os.path.join(d, o)) == w, o


def test_batch_tuning_reported(flats):
    with ab.Session(flats[0]) as s:
        s.execute_batch([wl.flat_script(i, out=f"t{i}.txt") for i in range(4)])
        cw, stages, bps = s.tuning()
        assert cw in (4, 8) and 2 <= stages <= 4 and bps >= 1


# ------------------------------------------------------- tables generated on the device

def _np_gen(seed, col, rows):
    """numpy restatement of the device generator (splitmix64 of seed, column, row)."""
    import numpy as np
    with np.errstate(over="ignore"):
        r = rows.astype(np.uint64)
        x = (np.uint64(seed) * np.uint64(0x100000001b3) + np.uint64(col) * np.uint64(0x9e3779b97f4a7c15)
             + r * np.uint64(0xd1b54a32d192ed03))
        z = x + np.uint64(0x9e3779b97f4a7c15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xbf58476d1ce4e5b9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94d049bb133111eb)
        h = z ^ (z >> np.uint64(31))
    if col == 1:
        return 1 + (h % np.uint64(50)).astype(np.int64)
    if col == 4:
        days = 8036 + (h % np.uint64(10561 - 8036 + 1)).astype(np.int64)
        return np.array([int(str(np.datetime64("1970-01-01") + np.timedelta64(int(d), "D")).replace("-", ""))
                         for d in days])
    if col == 5:
        return (h % np.uint64(3)).astype(np.int64)
    raise ValueError(col)


def test_device_generated_table_values_and_groupby():
    import tempfile
    import numpy as np
    segs = [100_000, 37, 250_001]
    n = sum(segs)
    rows = np.arange(n)
    qty, ship, flag = _np_gen(9, 1, rows), _np_gen(9, 4, rows), _np_gen(9, 5, rows)
    assert all(ab.lib().alk_gen_flat_value(9, c, 12345) == int(v[12345]) for c, v in ((1, qty), (4, ship), (5, flag)))
    cut = 19950617
    script = ("LF := FILTER gl BY l_shipdate < %d;\n"
              "R := SELECT l_returnflag AS f, SUM(l_quantity) AS q, COUNT(l_orderkey) AS c FROM LF "
              "GROUP BY l_returnflag;\nSTORE R INTO 'gr.txt' USING ('|');\n" % cut)
    outs = {}
    with tempfile.TemporaryDirectory() as d:
        for plain in (True, False):
            with ab.Session(d, plain=plain) as s:
                s.gen_flat_resident("gl", segs, 9)
                s.execute(script)
                assert s.stats().plan == (0 if plain else 1)
                outs[plain] = open(os.path.join(d, "gr.txt"), "rb").read()
    assert outs[True] == outs[False]
    got = {}
    for line in outs[True].decode().splitlines():
        f, q, c = line.split("|")[:3]
        got[f] = (int(q), int(c))
    m = ship < cut
    want = {k: (int(qty[m & (flag == i)].sum()), int((m & (flag == i)).sum())) for i, k in enumerate("ANR")}
    assert got == want


def test_batch_fixed_launch_shape(flats):
    d = flats[2]
    scripts = [wl.flat_script(40 + i, out=f"fx{i}.txt") for i in range(3)]
    want = []
    for i, sc in enumerate(scripts):
        _oracle.execute(d, sc.replace(f"fx{i}.txt", f"oracle_fx{i}.txt"))
        want.append(_read(os.path.join(d, f"oracle_fx{i}.txt")))
    with ab.Session(d) as s:
        with pytest.raises(ab.AlenkaError):
            s.set_tuning((5, 2, 1))  # 4 or 8 consumer warps only
        for shape in ((4, 2, 2), (8, 4, 1)):
            s.set_tuning(shape)
            s.execute_batch(scripts)
            assert s.tuning() == shape
            for i, w in enumerate(want):
                assert _read(os.path.join(d, f"fx{i}.txt")) == w


def test_batch_store_failures_and_shared_paths(flats):
    """The final STOREs of a batch are written after it: an unwritable path still fails
    its own script, and two scripts storing into one file leave the later one's rows."""
    d = flats[1]
    first = wl.flat_script(61, out="same.txt")
    second = wl.flat_script(62, out="same.txt")
    unwritable = wl.flat_script(63, out="no_such_dir/x.txt")
    other = wl.flat_script(64, out="o64.txt")
    _oracle.execute(d, second.replace("same.txt", "oracle_same.txt"))
    _oracle.execute(d, other.replace("o64.txt", "oracle_o64.txt"))
    with ab.Session(d) as s:
        with pytest.raises(ab.AlenkaError) as e:
            s.execute_batch([first, unwritable, second, other])
        assert "script 1" in str(e.value) and "Could not open file" in str(e.value)
    assert _read(os.path.join(d, "same.txt")) == _read(os.path.join(d, "oracle_same.txt"))
    assert _read(os.path.join(d, "o64.txt")) == _read(os.path.join(d, "oracle_o64.txt"))
