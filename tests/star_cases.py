"""Cases of the star join golden set (tests/golden/star): seeded three-way tables, the
bitmap join indexes a setup script creates on them, and star join scripts over those
indexes. tests/golden/make_star.py records what the reference itself writes for each
(the index files and the stored results); tests/test_star.py checks the oracle (CPU) and
the engine (GPU) against that.

Every dimension table here is one segment (the reference's CREATE INDEX reads the
dimension's first segment only). star_a keeps orders in one segment and lineitem in four,
so lineitem can be indexed on orders' columns and a star join can take two filtered views
of orders at once; star_b splits orders into three segments and lineitem into twelve."""

DATASETS = {
    "star_a": {"kind": "three_way", "customers": 1500, "orders": 15000, "rows": 60000, "seg_rows": 15000, "seed": 5},
    "star_b": {"kind": "three_way", "customers": 1500, "orders": 15000, "rows": 60000, "seg_rows": 5000, "seed": 7},
    # lineitem segments of 200 rows: l_orderkey is stored in 8 bits with values past 127,
    # which the star join reads through a signed char
    "star_c": {"kind": "three_way", "customers": 50, "orders": 200, "rows": 800, "seg_rows": 200, "seed": 3},
    # customer (6000 rows, one segment) longer than the last orders segment (3000 rows):
    # the char index appends the dimension's remaining hashes to that segment's values
    "star_d": {"kind": "three_way", "customers": 6000, "orders": 15000, "rows": 24000, "seg_rows": 6000, "seed": 9},
}

SETUP = {
    "star_a": (
        "CREATE INDEX lo ON lineitem(orders.o_orderdate) FROM lineitem, orders "
        "WHERE lineitem.l_orderkey = orders.o_orderkey;\n"
        "CREATE INDEX lp ON lineitem(orders.o_shippriority) FROM lineitem, orders "
        "WHERE lineitem.l_orderkey = orders.o_orderkey;\n"
        "CREATE INDEX oc ON orders(customer.c_mktsegment) FROM orders, customer "
        "WHERE orders.o_custkey = customer.c_custkey;\n"),
    "star_b": (
        "CREATE INDEX oc ON orders(customer.c_mktsegment) FROM orders, customer "
        "WHERE orders.o_custkey = customer.c_custkey;\n"),
    "star_c": (
        "CREATE INDEX lo ON lineitem(orders.o_orderdate) FROM lineitem, orders "
        "WHERE lineitem.l_orderkey = orders.o_orderkey;\n"),
    "star_d": (
        "CREATE INDEX oc ON orders(customer.c_mktsegment) FROM orders, customer "
        "WHERE orders.o_custkey = customer.c_custkey;\n"),
}

# the index files each setup writes (fact.dimension.column.segment)
INDEX_FILES = {
    "star_a": [f"lineitem.orders.{c}.{g}" for c in ("o_orderdate", "o_shippriority") for g in range(4)]
    + ["orders.customer.c_mktsegment.0"],
    "star_b": [f"orders.customer.c_mktsegment.{g}" for g in range(3)],
    "star_c": [f"lineitem.orders.o_orderdate.{g}" for g in range(4)],
    "star_d": [f"orders.customer.c_mktsegment.{g}" for g in range(3)],
}

CASES = [
    # two filtered views of one dimension: both filters move into the fact's, AND-ed
    {"name": "a_two_dims", "dataset": "star_a", "out": "a1.txt", "script": (
        "OF1 := FILTER orders BY o_orderdate == 19950315 OR o_orderdate == 19960102;\n"
        "OF2 := FILTER orders BY o_shippriority == 0;\n"
        "J := SELECT l_orderkey AS l_orderkey, l_shipdate AS l_shipdate, o_orderdate AS o_orderdate "
        "FROM lineitem JOIN OF1 ON l_orderkey = o_orderkey JOIN OF2 ON l_orderkey = o_orderkey;\n"
        "STORE J INTO 'a1.txt' USING ('|');\n")},
    # a filtered fact table, a number before the index column, fact and dimension columns
    {"name": "a_fact_filter", "dataset": "star_a", "out": "a2.txt", "script": (
        "LF := FILTER lineitem BY l_shipdate > 19960101;\n"
        "OF := FILTER orders BY 19950315 == o_orderdate OR o_orderdate == 19970601;\n"
        "J := SELECT l_orderkey AS l_orderkey, l_extendedprice AS l_extendedprice, l_discount AS l_discount, "
        "o_orderdate AS o_orderdate, o_custkey AS o_custkey FROM LF JOIN OF ON l_orderkey = o_orderkey;\n"
        "STORE J INTO 'a2.txt' USING ('|');\n")},
    # '<' on an index column keeps every code but the constant's (cmp_functor_dict); nearly
    # every row passes, so the last rows of segments hit the row-list quirk
    {"name": "a_less_than", "dataset": "star_a", "out": "a3.txt", "script": (
        "OF := FILTER orders BY o_orderdate < 19950315;\n"
        "J := SELECT l_orderkey AS l_orderkey, l_discount AS l_discount, o_orderdate AS o_orderdate "
        "FROM lineitem JOIN OF ON l_orderkey = o_orderkey;\n"
        "STORE J INTO 'a3.txt' USING ('|');\n")},
    # a char dimension column, then a GROUP BY over the star join's result
    {"name": "a_group_after", "dataset": "star_a", "out": "a4.txt", "script": (
        'CF := FILTER customer BY c_mktsegment == "BUILDING" OR c_mktsegment == "HOUSEHOLD";\n'
        "J := SELECT o_orderkey AS o_orderkey, o_orderdate AS o_orderdate, c_mktsegment AS c_mktsegment "
        "FROM orders JOIN CF ON o_custkey = c_custkey;\n"
        "G := SELECT c_mktsegment AS seg, COUNT(o_orderkey) AS cnt, MAX(o_orderdate) AS last "
        "FROM J GROUP BY c_mktsegment;\n"
        "STORE G INTO 'a4.txt' USING ('|');\n")},
    # a literal no dictionary holds: != keeps nothing
    {"name": "a_absent_literal", "dataset": "star_a", "out": "a5.txt", "script": (
        'CF := FILTER customer BY c_mktsegment != "NOSUCH";\n'
        "J := SELECT o_orderkey AS o_orderkey, c_mktsegment AS c_mktsegment "
        "FROM orders JOIN CF ON o_custkey = c_custkey;\n"
        "STORE J INTO 'a5.txt' USING ('|');\n")},
    # a dimension filter column without an index, in a join of two tables
    {"name": "a_missing_index", "dataset": "star_a", "out": "a6.txt", "script": (
        "OF1 := FILTER orders BY o_custkey == 5;\n"
        "OF2 := FILTER orders BY o_shippriority == 0;\n"
        "J := SELECT l_orderkey AS l_orderkey, o_orderdate AS o_orderdate "
        "FROM lineitem JOIN OF1 ON l_orderkey = o_orderkey JOIN OF2 ON l_orderkey = o_orderkey;\n"
        "STORE J INTO 'a6.txt' USING ('|');\n")},
    # three index segments; the dense customer keys meet the lower_bound of (key - 1)
    {"name": "b_segment", "dataset": "star_b", "out": "b1.txt", "script": (
        'CF := FILTER customer BY c_mktsegment == "BUILDING";\n'
        "J := SELECT o_orderkey AS o_orderkey, o_orderdate AS o_orderdate, c_mktsegment AS c_mktsegment "
        "FROM orders JOIN CF ON o_custkey = c_custkey;\n"
        "STORE J INTO 'b1.txt' USING ('|');\n")},
    {"name": "b_fact_filter_ne", "dataset": "star_b", "out": "b2.txt", "script": (
        "OF := FILTER orders BY o_orderdate < 19950101;\n"
        'CF := FILTER customer BY c_mktsegment != "MACHINERY";\n'
        "J := SELECT o_orderkey AS o_orderkey, c_mktsegment AS c_mktsegment, o_custkey AS o_custkey "
        "FROM OF JOIN CF ON o_custkey = c_custkey;\n"
        "STORE J INTO 'b2.txt' USING ('|');\n")},
    # fact columns only: l_orderkey's 8-bit stored values past 127 come back negative
    {"name": "c_signed_char", "dataset": "star_c", "out": "c1.txt", "script": (
        "OF := FILTER orders BY o_orderdate != 19951019 OR o_orderdate != 19950122 OR o_orderdate != 19930423 "
        "OR o_orderdate != 19950412;\n"
        "J := SELECT l_orderkey AS l_orderkey, l_extendedprice AS l_extendedprice, l_shipdate AS l_shipdate "
        "FROM lineitem JOIN OF ON l_orderkey = o_orderkey;\n"
        "STORE J INTO 'c1.txt' USING ('|');\n")},
]


def make_dataset(d, ds, gen):
    gen.three_way(d, ds["customers"], ds["orders"], ds["rows"], ds["seg_rows"], ds["seed"])
