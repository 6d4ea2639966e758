"""ORDER BY on char columns against the oracle, byte for byte. The reference sorts the
rows' strings (unsigned bytes over the full column width, stable; descending by the
reversed comparison): update_char_permutation (cm.cu:4218) with str_sort
(strings_sort_device.cu:125). The engine sorts by each code's rank in the byte-ordered
dictionary, which must give the same rows in the same order, ties included."""
import os

import pytest

import alenka_b200 as ab

from . import _oracle
from .test_gpu_parity import _read

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def names(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("names_order"))
    ab.gen_names(d, 120_000, 1_500, 50_000, 13)
    return d


ORDERS = [
    ("NF := FILTER names BY n_key > 100;\n"
     "R := SELECT n_name AS nm, COUNT(n_key) AS c FROM NF GROUP BY n_name;\n"
     "S := ORDER R BY nm {d};\n"),
    ("NF := FILTER names BY n_key > 100;\n"
     "R := SELECT n_name AS nm, COUNT(n_key) AS c FROM NF GROUP BY n_name;\n"
     "S := ORDER R BY c DESC, nm {d};\n"),
    ("NF := FILTER names BY n_key < 30000;\n"
     "R := SELECT n_key AS k, n_name AS nm FROM NF;\n"
     "S := ORDER R BY nm {d}, k DESC;\n"),
    ("NF := FILTER names BY n_name LIKE \"%.%\";\n"
     "R := SELECT n_key AS k, n_name AS nm FROM NF;\n"
     "S := ORDER R BY nm {d};\n"),
]


@pytest.mark.parametrize("direction", ["ASC", "DESC"])
@pytest.mark.parametrize("which", range(len(ORDERS)))
def test_order_by_char_matches_oracle(names, which, direction):
    script = ORDERS[which].format(d=direction) + "STORE S INTO 'ord.txt' USING ('|') LIMIT 5000;\n"
    _oracle.execute(names, script.replace("ord.txt", "oracle_ord.txt"))
    want = _read(os.path.join(names, "oracle_ord.txt"))
    for plain in (False, True):
        with ab.Session(names, plain=plain) as s:
            s.execute(script)
        assert _read(os.path.join(names, "ord.txt")) == want, plain
    assert want
