"""Cases of the reference-pinned golden set (tests/golden/ref_ops): seeded tables and the
scripts run over them. tests/golden/make_ref_ops.py records what the reference itself
stores for each; tests/test_ref_golden.py checks the oracle and the engine against that.

The tables come from oracle/refdata.py (or, on a GPU box, the product's generators,
which write the same bytes); their digest is part of the manifest. Scripts are literal
text with seed-drawn constants, in the shapes of the benchmark workloads: the
single-table FILTER + GROUP BY (config 1, also at its stated 6M rows), the three-way
FILTER -> JOIN -> JOIN -> GROUP BY -> ORDER of the reference's README (config 2, also at
its stated 60M / 15M / 1.5M rows, and at the benchmark's 600M / 150M / 15M), and operator
scripts around them."""
import random

SEGMENTS = ["AUTOMOBILE", "BUILDING", "FURNITURE", "HOUSEHOLD", "MACHINERY"]


def _date_add_days(v, days):
    from oracle import refdata
    return refdata.date_add_days(v, days)


DATASETS = {
    # name: generator, its arguments, and the fact rows
    "flat_multi": {"kind": "flat", "rows": 300_000, "seg_rows": 100_000, "seed": 11},
    "flat_single": {"kind": "flat", "rows": 250_000, "seg_rows": 0, "seed": 12},
    "three_way": {"kind": "three_way", "customers": 15_000, "orders": 150_000, "rows": 600_000,
                  "seg_rows": 200_000, "seed": 5},
    "config1": {"kind": "flat", "rows": 6_000_000, "seg_rows": 2_000_000, "seed": 1},
    "config2": {"kind": "three_way", "customers": 1_500_000, "orders": 15_000_000, "rows": 60_000_000,
                "seg_rows": 10_000_000, "seed": 1},
    # the headline instance: the three-way pipeline at lineitem 600M / orders 150M /
    # customer 15M (the benchmark's default tables)
    "headline600": {"kind": "three_way", "customers": 15_000_000, "orders": 150_000_000, "rows": 600_000_000,
                    "seg_rows": 10_000_000, "seed": 1},
}


def make_dataset(d, ds, gen):
    """Writes dataset ds into directory d with gen: oracle.refdata (numpy) or an object with
    the same two functions over the product's generators."""
    if ds["kind"] == "flat":
        gen.lineitem_flat(d, ds["rows"], ds["seg_rows"], ds["seed"])
    else:
        gen.three_way(d, ds["customers"], ds["orders"], ds["rows"], ds["seg_rows"], ds["seed"])


def flat_script(seed, out):
    cut = _date_add_days(19950617, random.Random(seed).randint(-30, 30))
    return (f"LF := FILTER lineitem BY l_shipdate < {cut};\n"
            "R := SELECT l_returnflag AS l_returnflag, l_linestatus AS l_linestatus, "
            "SUM(l_quantity) AS sum_qty, SUM(l_extendedprice) AS sum_base_price, "
            "SUM(l_extendedprice*(1-l_discount)) AS sum_disc_price, COUNT(l_orderkey) AS count_order "
            "FROM LF GROUP BY l_returnflag, l_linestatus;\n"
            f"STORE R INTO '{out}' USING ('|');\n")


def three_way_with(lf, of, cf, out, limit=10):
    lim = f" LIMIT {limit}" if limit else ""
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
            f"STORE RES INTO '{out}' USING ('|'){lim};\n")


def three_way_script(seed, out, limit=10):
    r = random.Random(seed * 7919 + 1)
    date = _date_add_days(19950702, r.randint(-30, 30))
    seg = SEGMENTS[r.randint(0, 4)]
    return three_way_with(f"l_shipdate > {date}", f"o_orderdate < {date}", f'c_mktsegment == "{seg}"', out, limit)


def random_three_way(seed, out):
    """Seeded operators and constants on all three tables."""
    r = random.Random(seed * 104729 + 3)
    ops = ["<", "<=", ">", ">="]
    ld = _date_add_days(19920102, r.randint(0, 2540))
    od = _date_add_days(19920102, r.randint(0, 2540))
    lf = f"l_shipdate {r.choice(ops)} {ld}"
    if r.random() < 0.5:
        lf += f" AND l_discount {r.choice(ops)} {r.randint(0, 10) / 100:.2f}"
    of = f"o_orderdate {r.choice(ops)} {od}"
    cf = f"c_mktsegment {r.choice(['==', '!='])} \"{SEGMENTS[r.randint(0, 4)]}\""
    return three_way_with(lf, of, cf, out)


SCRIPTS = {
    "and_or_decimal": (
        "LF := FILTER lineitem BY l_shipdate >= 19940101 AND l_quantity < 25 OR l_discount == 0.05;\n"
        "R := SELECT l_returnflag AS f, l_linestatus AS s, AVG(l_quantity) AS aq, MIN(l_extendedprice) AS mn, "
        "MAX(l_extendedprice) AS mx, COUNT(l_orderkey) AS c FROM LF GROUP BY l_returnflag, l_linestatus;\n"
        "STORE R INTO 'x.txt' USING ('|');\n"),
    "one_line": (
        "LF := FILTER lineitem BY l_shipdate < 19960101;\n"
        "S := SELECT SUM(l_quantity) AS q, COUNT(l_orderkey) AS c, MIN(l_extendedprice) AS mn, "
        "MAX(l_extendedprice) AS mx, AVG(l_quantity) AS a FROM LF;\n"
        "STORE S INTO 'x.txt' USING (',');\n"),
    "projection_order": (
        "LF := FILTER lineitem BY l_shipdate > 19980601;\n"
        "P := SELECT l_orderkey AS k, l_extendedprice*(1-l_discount) AS rev, l_shipdate AS d FROM LF;\n"
        "O := ORDER P BY rev DESC, d ASC;\n"
        "STORE O INTO 'x.txt' USING ('|') LIMIT 200;\n"),
    "strings": (
        "F := FILTER lineitem BY l_returnflag == \"R\" AND l_linestatus != \"O\";\n"
        "R := SELECT l_returnflag AS f, l_linestatus AS s, SUM(l_quantity) AS q, COUNT(l_orderkey) AS c "
        "FROM F GROUP BY l_returnflag, l_linestatus;\n"
        "STORE R INTO 'x.txt' USING ('|');\n"),
    "filter_arith": (
        "F := FILTER lineitem BY l_quantity*2 > 60 AND l_extendedprice - 1000.00 < 50000.00;\n"
        "R := SELECT l_linestatus AS s, SUM(l_extendedprice) AS p, COUNT(l_orderkey) AS c FROM F GROUP BY l_linestatus;\n"
        "STORE R INTO 'x.txt' USING ('|');\n"),
    "chained_filter_keys": (
        "F := FILTER lineitem BY l_shipdate < 19970101;\n"
        "G := FILTER F BY l_quantity > 10;\n"
        "R := SELECT l_orderkey AS k, SUM(l_quantity) AS q, COUNT(l_orderkey) AS c FROM G GROUP BY l_orderkey;\n"
        "O := ORDER R BY q DESC;\n"
        "STORE O INTO 'x.txt' USING ('|') LIMIT 100;\n"),
    "empty_filter": (
        "F := FILTER lineitem BY l_shipdate < 19000101;\n"
        "R := SELECT l_linestatus AS s, COUNT(l_orderkey) AS c FROM F GROUP BY l_linestatus;\n"
        "STORE R INTO 'x.txt' USING ('|');\n"),
    "min_max_avg_keys": (
        "F := FILTER lineitem BY l_discount >= 0.04 AND l_discount <= 0.06;\n"
        "R := SELECT l_linestatus AS s, l_returnflag AS f, MIN(l_quantity) AS mnq, MAX(l_shipdate) AS mxd, "
        "AVG(l_extendedprice) AS ap, SUM(l_discount) AS sd, COUNT(l_orderkey) AS c FROM F "
        "GROUP BY l_linestatus, l_returnflag;\n"
        "STORE R INTO 'x.txt' USING ('|');\n"),
}

# Zone maps over the segments of flat_multi (l_orderkey in order: [1, 24789],
# [24789, 49806], [49807, 74916]): each filter gives the three segments different
# verdicts (zone_map.cu:720-1135); name -> (script, segments the verdicts skip)
ZONE_SCRIPTS = {
    "zone_n_r_a": (
        "LF := FILTER lineitem BY l_orderkey > 30000 AND l_orderkey < 80000;\n"
        "R := SELECT l_returnflag AS f, l_linestatus AS s, SUM(l_quantity) AS q, COUNT(l_orderkey) AS c "
        "FROM LF GROUP BY l_returnflag, l_linestatus;\n"
        "STORE R INTO 'z.txt' USING ('|');\n", 1),
    "zone_r_r_n": (
        "LF := FILTER lineitem BY l_orderkey >= 24789 AND l_orderkey <= 24789;\n"
        "R := SELECT l_orderkey AS k, SUM(l_extendedprice) AS p, COUNT(l_orderkey) AS c FROM LF GROUP BY l_orderkey;\n"
        "STORE R INTO 'z.txt' USING ('|');\n", 1),
    "zone_r_n_n_or": (
        "LF := FILTER lineitem BY l_orderkey < 24789 OR l_orderkey > 90000;\n"
        "R := SELECT l_linestatus AS s, SUM(l_quantity) AS q, COUNT(l_orderkey) AS c FROM LF GROUP BY l_linestatus;\n"
        "STORE R INTO 'z.txt' USING ('|');\n", 2),
}

FUSED_PREDICATES = {
    "ge_le": ("l_shipdate >= 19950315", "o_orderdate <= 19950315", 'c_mktsegment == "BUILDING"'),
    "eq_ne": ("l_shipdate == 19950320", "o_orderdate != 19950301", 'c_mktsegment != "MACHINERY"'),
    "always": ("l_shipdate > 19000101", "o_orderdate < 20500101", 'c_mktsegment != "NOSUCHSEG"'),
    "never_fact": ("l_shipdate < 19000101", "o_orderdate < 19960101", 'c_mktsegment == "HOUSEHOLD"'),
    "never_dim": ("l_shipdate > 19940101", "o_orderdate > 20500101", 'c_mktsegment == "HOUSEHOLD"'),
    "decimal": ("l_discount > 0.05 AND l_extendedprice < 60000.00", "o_orderdate > 19960101 AND o_orderdate < 19970101",
                'c_mktsegment == "FURNITURE"'),
    "disjunction": ("l_shipdate < 19930301 OR l_shipdate > 19980101", "o_orderdate < 19930101 OR o_orderdate > 19971001",
                    'c_mktsegment == "AUTOMOBILE" OR c_mktsegment == "BUILDING"'),
    "three_conj": ("l_shipdate > 19950101 AND l_shipdate < 19950601 AND l_discount <= 0.03",
                   "o_orderdate >= 19941001", 'c_mktsegment == "BUILDING"'),
}

# emit_multijoin's other forms (operators.cu:1288-1399); left rows come in left order and
# right rows in key order, so those outputs are compared byte for byte
_JF = ("OFI := FILTER orders BY o_orderdate < 19950101;\n"
       "LF := FILTER lineitem BY l_shipdate < 19950301;\n")
JOIN_FORMS = {
    "and_same_pair": (_JF + "J := SELECT l_orderkey AS lk, o_orderdate AS od FROM LF JOIN OFI "
                            "ON l_orderkey = o_orderkey AND l_orderkey = o_orderkey;\n"
                            "STORE J INTO 'jf.txt' USING ('|');\n", "multiset"),
    "and_second_pair": (_JF + "J := SELECT l_orderkey AS lk, l_discount AS d, o_orderdate AS od FROM LF JOIN OFI "
                              "ON l_orderkey = o_orderkey AND l_discount = o_shippriority;\n"
                              "STORE J INTO 'jf.txt' USING ('|');\n", "multiset"),
    "left_semi": (_JF + "K := SELECT l_orderkey AS lk, l_extendedprice AS p FROM LF LEFT SEMI JOIN OFI "
                        "ON l_orderkey = o_orderkey;\n"
                        "STORE K INTO 'jf.txt' USING ('|');\n", "bytes"),
    "left_semi_and": (_JF + "K := SELECT l_orderkey AS lk, l_shipdate AS sd FROM LF LEFT SEMI JOIN OFI "
                            "ON l_orderkey = o_orderkey AND l_discount = o_shippriority;\n"
                            "STORE K INTO 'jf.txt' USING ('|');\n", "bytes"),
    "left_anti": (_JF + "M := SELECT l_orderkey AS lk, l_shipdate AS sd FROM LF LEFT ANTI JOIN OFI "
                        "ON l_orderkey = o_orderkey;\n"
                        "STORE M INTO 'jf.txt' USING ('|');\n", "bytes"),
    "right_semi": (_JF + "R := SELECT o_orderkey AS ok, o_orderdate AS od FROM LF RIGHT SEMI JOIN OFI "
                         "ON l_orderkey = o_orderkey;\n"
                         "STORE R INTO 'jf.txt' USING ('|');\n", "bytes"),
    "right_anti": (_JF + "RA := SELECT o_orderkey AS ok, o_custkey AS ck FROM LF RIGHT ANTI JOIN OFI "
                         "ON l_orderkey = o_orderkey;\n"
                         "STORE RA INTO 'jf.txt' USING ('|');\n", "bytes"),
    "left_semi_grouped": (_JF + "K := SELECT l_orderkey AS lk, l_extendedprice AS p FROM LF LEFT SEMI JOIN OFI "
                                "ON l_orderkey = o_orderkey;\n"
                                "G := SELECT lk AS k, SUM(p) AS s, COUNT(lk) AS c FROM K GROUP BY lk;\n"
                                "O := ORDER G BY s DESC, k ASC;\n"
                                "STORE O INTO 'jf.txt' USING ('|') LIMIT 20;\n", "bytes"),
}

JOIN_SCRIPTS = {
    # join output with no ORDER: the reference's row order comes from its sort-merge, so
    # it is compared as a multiset
    "join_two_way_multiset": (
        "OFI := FILTER orders BY o_orderdate < 19950101;\n"
        "CF := FILTER customer BY c_mktsegment == \"BUILDING\";\n"
        "J := SELECT o_orderkey AS ok, o_orderdate AS od, c_custkey AS ck FROM OFI JOIN CF ON o_custkey = c_custkey;\n"
        "STORE J INTO 'j.txt' USING ('|');\n", "j.txt", "multiset"),
    # a decimal column kept under its own name keeps its scale; the aliased one does not
    "join_alias_scale": (
        "LF := FILTER lineitem BY l_shipdate > 19950611;\n"
        "OFI := FILTER orders BY o_orderdate < 19950611;\n"
        "J := SELECT o_orderkey AS o_orderkey, l_extendedprice AS l_extendedprice, l_discount AS discount "
        "FROM LF JOIN OFI ON l_orderkey = o_orderkey;\n"
        "F := SELECT o_orderkey AS k, SUM(l_extendedprice*(1-discount)) AS rev, SUM(l_extendedprice) AS sp, "
        "COUNT(o_orderkey) AS c FROM J GROUP BY o_orderkey;\n"
        "O := ORDER F BY rev ASC, k ASC;\n"
        "STORE O INTO 'j.txt' USING ('|') LIMIT 50;\n", "j.txt", "bytes"),
    "join_projection_multiset": (
        "LF := FILTER lineitem BY l_shipdate > 19980101;\n"
        "OFI := FILTER orders BY o_orderdate > 19971101;\n"
        "J := SELECT l_orderkey AS lk, o_orderdate AS od, l_extendedprice AS price FROM LF JOIN OFI ON l_orderkey = o_orderkey;\n"
        "STORE J INTO 'j.txt' USING ('|');\n", "j.txt", "multiset"),
}


def _cases():
    c = []
    for seed in (1, 2, 3):
        c.append({"name": f"flat_multi_q1_s{seed}", "dataset": "flat_multi", "script": flat_script(seed, "q1.txt"),
                  "out": "q1.txt"})
    c.append({"name": "flat_single_q1_s4", "dataset": "flat_single", "script": flat_script(4, "q1.txt"), "out": "q1.txt"})
    for ds in ("flat_multi", "flat_single"):
        for n, sc in sorted(SCRIPTS.items()):
            c.append({"name": f"{ds}_{n}", "dataset": ds, "script": sc, "out": "x.txt"})
    for seed in (1, 2):
        c.append({"name": f"three_way_q3_s{seed}", "dataset": "three_way", "script": three_way_script(seed, "q3.txt"),
                  "out": "q3.txt"})
    c.append({"name": "three_way_q3_all_groups", "dataset": "three_way",
              "script": three_way_script(4, "q3.txt", limit=0), "out": "q3.txt"})
    for n, p in sorted(FUSED_PREDICATES.items()):
        c.append({"name": f"three_way_fused_{n}", "dataset": "three_way", "script": three_way_with(*p, "fx.txt"),
                  "out": "fx.txt"})
    c.append({"name": "three_way_fused_decimal_all_groups", "dataset": "three_way",
              "script": three_way_with(*FUSED_PREDICATES["decimal"], "fx.txt", limit=0), "out": "fx.txt"})
    for seed in range(1, 7):
        c.append({"name": f"three_way_random_s{seed}", "dataset": "three_way", "script": random_three_way(seed, "qr.txt"),
                  "out": "qr.txt"})
    for n, (sc, skipped) in sorted(ZONE_SCRIPTS.items()):
        c.append({"name": f"flat_multi_{n}", "dataset": "flat_multi", "script": sc, "out": "z.txt",
                  "segments_skipped": skipped})
    # the fused three-way plan with a fact filter whose zone maps skip two of the three
    # lineitem segments ([4, 200392], [200392, 400024], [400024, 599664])
    c.append({"name": "three_way_zone_fact_skip", "dataset": "three_way",
              "script": three_way_with("l_orderkey < 200000 AND l_shipdate > 19950101", "o_orderdate < 19960101",
                                       'c_mktsegment == "BUILDING"', "fx.txt", limit=0),
              "out": "fx.txt", "segments_skipped": 2})
    for n, (sc, mode) in sorted(JOIN_FORMS.items()):
        c.append({"name": f"three_way_join_{n}", "dataset": "three_way", "script": sc, "out": "jf.txt", "mode": mode})
    for n, (sc, out, mode) in sorted(JOIN_SCRIPTS.items()):
        c.append({"name": f"three_way_{n}", "dataset": "three_way", "script": sc, "out": out, "mode": mode})
    # the stated sizes: config 1 (6M rows) and config 2 (60M / 15M / 1.5M)
    c.append({"name": "config1_q1_s1", "dataset": "config1", "script": flat_script(1, "q1.txt"), "out": "q1.txt"})
    c.append({"name": "config2_q3_s1", "dataset": "config2", "script": three_way_script(1, "q3.txt"), "out": "q3.txt"})
    c.append({"name": "config2_q3_all_groups", "dataset": "config2", "script": three_way_script(1, "q3.txt", limit=0),
              "out": "q3.txt"})
    c.append({"name": "headline600_q3_s1", "dataset": "headline600", "script": three_way_script(1, "q3.txt"),
              "out": "q3.txt"})
    return c


CASES = _cases()
