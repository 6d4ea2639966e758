"""Text files and LOAD scripts for the text loader (LOAD ... USING (sep) AS (...), then
STORE ... BINARY and a query over the stored table). The files carry the forms the
reference's parse functors treat specially: signs and leading spaces, decimals with
fewer and more fraction digits than the declared scale, dates, a quoted field holding
the separator, declared columns out of field order and a decimal of scale 0."""
import random

CASES = {}


def _numeric_text(seed, rows):
    r = random.Random(seed)
    lines = []
    for i in range(rows):
        a = r.randint(-10**6, 10**6)
        a_txt = (" " * r.randint(0, 2)) + ("+" if a >= 0 and r.random() < 0.1 else "") + str(a)
        whole = r.randint(-99999, 99999)
        frac_digits = r.choice([0, 1, 2, 3, 4])
        p_txt = str(whole) + ("." + "".join(str(r.randint(0, 9)) for _ in range(frac_digits)) if frac_digits else "")
        if whole == 0 and r.random() < 0.5:
            p_txt = "-0." + "".join(str(r.randint(0, 9)) for _ in range(2))
        d_txt = f"{r.randint(1992, 1998)}-{r.randint(1, 12):02d}-{r.randint(1, 28):02d}"
        q_txt = '"x|' + "".join(r.choice("abc|") for _ in range(r.randint(0, 5))) + '"'
        b = r.randint(0, 500)
        s = r.randint(1, 999)
        lines.append(f"{a_txt}|{p_txt}|{d_txt}|{q_txt}|{b}|{s}|")
    return "\n".join(lines) + "\n"


CASES["numeric"] = {
    "text": lambda: _numeric_text(7, 5000),
    # the stored table is queried by a second script (a script's first pass checks its
    # sources against the catalog, where the STORE has not yet put the table)
    "scripts": ["T := LOAD 'numeric.tbl' USING ('|') AS (a{1}:int, p{2}:decimal(12,2), d{3}:int, b{5}:int, "
                "s{6}:decimal(5,0));\n"
                "STORE T INTO 'tnum' BINARY;\n",
                "F := FILTER tnum BY b < 250;\n"
                "R := SELECT b AS b, SUM(p) AS sp, MIN(d) AS md, MAX(a) AS ma, SUM(s) AS ss, COUNT(a) AS c "
                "FROM F GROUP BY b;\n"
                "STORE R INTO 'tnum_q.txt' USING ('|');\n"],
    "table": "tnum",
}
CASES["field_order"] = {
    # declared out of field order: declared column i reads the i-th smallest field
    "text": lambda: _numeric_text(8, 1200),
    "scripts": ["T := LOAD 'order.tbl' USING ('|') AS (x{5}:int, y{1}:int, z{6}:int);\n"
                "STORE T INTO 'tord' BINARY;\n"],
    "table": "tord",
}
def _char_text(seed, rows):
    r = random.Random(seed)
    # quoted values keep their quotes: every value, quotes included, fits the 12-byte width
    # (a longer one runs past its slot into the next record's in the reference, an
    # overflow whose outcome depends on the order its threads take the records)
    names = ["alpha", "beta", "gamma|x", "delta", "", "omega-name", "zeta"]
    lines = []
    for i in range(rows):
        flag = r.choice("ANR")
        nm = r.choice(names)
        nm_txt = f'"{nm}"' if "|" in nm or r.random() < 0.2 else nm
        code = "".join(r.choice("XYZ") for _ in range(r.randint(1, 9)))
        lines.append(f"{i + 1}|{flag}|{nm_txt}|{r.randint(1, 50)}|{code}|")
    return "\n".join(lines) + "\n"


CASES["chars"] = {
    # char columns: a flag, names (quoted ones hold the separator; the quotes stay in
    # the value), a NO ENCODING column
    "text": lambda: _char_text(10, 3000),
    "scripts": ["T := LOAD 'chars.tbl' USING ('|') AS (k{1}:int, f{2}:varchar(1), nm{3}:varchar(12), "
                "q{4}:int, cd{5}:varchar(8) NO ENCODING);\n"
                "STORE T INTO 'tch' BINARY;\n",
                "F := FILTER tch BY q > 10;\n"
                "R := SELECT f AS f, nm AS nm, SUM(q) AS sq, COUNT(k) AS c FROM F GROUP BY f, nm;\n"
                "STORE R INTO 'tch_q.txt' USING ('|');\n"],
    "table": "tch",
}


# A file whose last line has no newline: the reference counts 299 records of 300 lines
# and then aborts in free() (invalid pointer), so there is no golden output for it; the
# engine's record count for it is tested on its own.
FILES = {"numeric": "numeric.tbl", "field_order": "order.tbl", "chars": "chars.tbl"}
