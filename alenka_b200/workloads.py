"""Benchmark and parity workloads: seeded synthetic tables of the TPC-H-like shapes and
the Alenka scripts run over them (single-table filter + group-by; the three-way
filter -> join -> group-by -> order pipeline of the reference's README)."""
import random

from . import date_add_days, gen_lineitem_flat, gen_three_way

SEGMENTS = ["AUTOMOBILE", "BUILDING", "FURNITURE", "HOUSEHOLD", "MACHINERY"]


def flat_cutoff(seed):
    """Shipdate cutoff near the median of 1992-01-02..1998-12-01 (about 50% selectivity)."""
    return date_add_days(19950617, random.Random(seed).randint(-30, 30))


def flat_script(seed, out="q1.txt", table="lineitem"):
    cut = flat_cutoff(seed)
    return (f"LF := FILTER {table} BY l_shipdate < {cut};\n"
            "R := SELECT l_returnflag AS l_returnflag, l_linestatus AS l_linestatus, "
            "SUM(l_quantity) AS sum_qty, SUM(l_extendedprice) AS sum_base_price, "
            "SUM(l_extendedprice*(1-l_discount)) AS sum_disc_price, COUNT(l_orderkey) AS count_order "
            "FROM LF GROUP BY l_returnflag, l_linestatus;\n"
            f"STORE R INTO '{out}' USING ('|');\n")


def three_way_params(seed):
    r = random.Random(seed * 7919 + 1)
    date = date_add_days(19950702, r.randint(-30, 30))
    return date, SEGMENTS[r.randint(0, 4)]


def three_way_script(seed, out="q3.txt", limit=10):
    date, seg = three_way_params(seed)
    lim = f" LIMIT {limit}" if limit else ""
    return (f"OFI := FILTER orders BY o_orderdate < {date};\n"
            f"CF := FILTER customer BY c_mktsegment == \"{seg}\";\n"
            f"LF := FILTER lineitem BY l_shipdate > {date};\n"
            "OLC := SELECT o_orderkey AS o_orderkey, o_orderdate AS o_orderdate, "
            "o_shippriority AS o_shippriority, l_extendedprice AS price, l_discount AS discount "
            "FROM LF JOIN OFI ON l_orderkey = o_orderkey JOIN CF ON o_custkey = c_custkey;\n"
            "F := SELECT o_orderkey AS o_orderkey1, o_orderdate AS orderdate1, o_shippriority AS priority, "
            "SUM(price*(1-discount)) AS sum_revenue, COUNT(o_orderkey) AS cnt "
            "FROM OLC GROUP BY o_orderkey, o_orderdate, o_shippriority;\n"
            "RES := ORDER F BY sum_revenue DESC, orderdate1 ASC;\n"
            f"STORE RES INTO '{out}' USING ('|'){lim};\n")


def card_script(seed, out="qc.txt"):
    """A three-way query of the README shape with seeded comparison operators and
    constants on all three tables (the estimator's training and test queries): dates
    anywhere in the 7-year range, any of <, <=, >, >=, sometimes a second lineitem
    conjunct on the discount, and == or != on the market segment."""
    r = random.Random(seed * 104729 + 3)
    ops = ["<", "<=", ">", ">="]
    ld = date_add_days(19920102, r.randint(0, 2540))
    od = date_add_days(19920102, r.randint(0, 2540))
    lf = f"l_shipdate {r.choice(ops)} {ld}"
    if r.random() < 0.3:
        lf += f" AND l_discount {r.choice(ops)} {r.randint(0, 10) / 100:.2f}"
    of = f"o_orderdate {r.choice(ops)} {od}"
    cf = f"c_mktsegment {r.choice(['==', '!='])} \"{SEGMENTS[r.randint(0, 4)]}\""
    return (f"OFI := FILTER orders BY {of};\n"
            f"CF := FILTER customer BY {cf};\n"
            f"LF := FILTER lineitem BY {lf};\n"
            "OLC := SELECT o_orderkey AS o_orderkey, o_orderdate AS o_orderdate, "
            "o_shippriority AS o_shippriority, l_extendedprice AS price, l_discount AS discount "
            "FROM LF JOIN OFI ON l_orderkey = o_orderkey JOIN CF ON o_custkey = c_custkey;\n"
            "F := SELECT o_orderkey AS o_orderkey1, o_orderdate AS orderdate1, o_shippriority AS priority, "
            "SUM(price*(1-discount)) AS sum_revenue, COUNT(o_orderkey) AS cnt "
            "FROM OLC GROUP BY o_orderkey, o_orderdate, o_shippriority;\n"
            "RES := ORDER F BY sum_revenue DESC, orderdate1 ASC;\n"
            f"STORE RES INTO '{out}' USING ('|') LIMIT 10;\n")


def batched_layout(queries=256, total_rows=6_000_000_000, seed=1, median=4_000_000, sigma=1.0,
                   lo=1_000_000, hi=32_000_000):
    """Segment sizes of the batched workload: lognormal (median 4M rows, clipped to
    [1M, 32M]) drawn until the total is reached, dealt to the queries' tables in turn.
    Returns one list of segment sizes per query (empty when the total ran out first)."""
    import math
    r = random.Random(seed * 7 + 5)
    tables = [[] for _ in range(queries)]
    total, i = 0, 0
    while total < total_rows:
        n = int(min(hi, max(lo, math.exp(math.log(median) + sigma * r.gauss(0.0, 1.0)))))
        n = min(n, total_rows - total)
        tables[i % queries].append(n)
        total += n
        i += 1
    return tables


# Full-size shapes (rows): the single-table workload and the three-way pipeline.
FLAT_ROWS = 6_000_000
THREE_WAY = dict(customers=1_500_000, orders=15_000_000, lineitems=60_000_000)


def make_flat(data_dir, rows=FLAT_ROWS, seg_rows=2_000_000, seed=1, delta=False):
    gen_lineitem_flat(data_dir, rows, seg_rows, seed, delta)


def make_three_way(data_dir, scale=1.0, seg_rows=10_000_000, seed=1, delta=False, zipf=0.0):
    """The three-way tables at scale (x the config-2 sizes). The compressed config stores
    them FOR-delta (delta=True) with Zipf(1.1) join keys (zipf=1.1)."""
    c = max(1, int(THREE_WAY["customers"] * scale))
    o = max(1, int(THREE_WAY["orders"] * scale))
    li = max(1, int(THREE_WAY["lineitems"] * scale))
    gen_three_way(data_dir, c, o, li, seg_rows, seed, delta, zipf)
    return li
