"""CPU restatement of the reference's text loader (test infrastructure: the oracle for
LOAD ... USING (sep) AS (...)), following CudaSet::LoadBigFile (cm.cu:1852-2080) and its
functors: parse_functor (cm.h:599-650), gpu_atoll (cm.h:543-597), gpu_atold
(cm.h:480-541) and gpu_date (cm.h:341-371). Pure Python, for small files.

Records are the newline-terminated lines. Declared column i reads the i-th smallest of
the declared field numbers. A field runs to the separator outside double quotes (the
quotes stay, NUL bytes are dropped) and is cut to a zero-filled 23-byte slot. A column
whose first record's slot has '-' at offset 4 is read as yyyy-mm-dd dates."""

SLOT = 23


def _cut(text, pos, sep, fields, widths=None):
    """The slots of the requested 0-based fields (ascending) of the record at pos: the
    field's bytes, NUL bytes dropped, cut or zero-padded to the slot's width (23 bytes,
    or widths[i])."""
    out, cur, want, j, quoted, n = [], 0, 0, pos, False, len(text)
    while want < len(fields):
        keep = fields[want] == cur
        w = widths[want] if widths else SLOT
        slot = bytearray(w)
        t = 0
        while j < n and (text[j] != sep or quoted):
            ch = text[j]
            if ch == 0x22:
                quoted = not quoted
            if keep and ch != 0 and t < w:
                slot[t] = ch
                t += 1
            j += 1
        j += 1
        if keep:
            out.append(bytes(slot))
            want += 1
        cur += 1
    return out


def _wrap(v):
    v &= (1 << 64) - 1
    return v - (1 << 64) if v >> 63 else v


def _sign_start(s):
    i = 0
    while i < SLOT and s[i] == 0x20:
        i += 1
    neg = False
    if i < SLOT and s[i] in (0x2D, 0x2B):
        neg = s[i] == 0x2D
        i += 1
    return i, neg


def parse_int(s):
    i, neg = _sign_start(s)
    acc = 0
    while i < SLOT and 0x30 <= s[i] <= 0x39:
        acc = acc * 10 - (s[i] - 0x30) if neg else acc * 10 + (s[i] - 0x30)
        i += 1
    return _wrap(acc)


def parse_decimal(s, scale):
    i, neg = _sign_start(s)
    acc, point, frac = 0, 0, False
    while i < SLOT:
        c = s[i]
        if 0x30 <= c <= 0x39:
            acc = acc * 10 - (c - 0x30) if neg else acc * 10 + (c - 0x30)
            if frac:
                point += 1
            if point == scale:
                break
        elif c == 0x2E:
            frac = True
        else:
            break
        i += 1
    return _wrap(acc * 10 ** (scale - point))


def parse_date(s):
    acc = 0
    for z in range(10):
        if s[z] != 0x2D:
            acc = acc * 10 + (s[z] - 0x30)
    return _wrap(acc)


def load(text, sep, cols):
    """cols: [(field (1-based), kind 'int' | 'decimal' | 'char', scale or width)] in
    declared order. Returns one list per declared column: int64 values, or the char
    column's width-byte values."""
    sepb = sep.encode()[0] if isinstance(sep, str) else sep
    fields = sorted(f - 1 for f, _, _ in cols)
    starts, p = [], 0
    for i, ch in enumerate(text):
        if ch == 0x0A:
            starts.append(p)
            p = i + 1
    if not starts:
        return [[] for _ in cols]
    widths = [scale if kind == "char" else SLOT for _, kind, scale in cols]
    first = _cut(text, 0, sepb, fields, widths)
    date = [cols[i][1] != "char" and first[i][4] == 0x2D for i in range(len(cols))]
    out = [[] for _ in cols]
    for st in starts:
        slots = _cut(text, st, sepb, fields, widths)
        for i, (_, kind, scale) in enumerate(cols):
            s = slots[i]
            if kind == "char":
                out[i].append(s)
            else:
                out[i].append(parse_date(s) if date[i] else parse_decimal(s, scale) if kind == "decimal"
                              else parse_int(s))
    return out
