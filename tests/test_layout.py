"""The generated C header agrees with the Python layout and parameter tables."""
import os

from ibis_b200 import layout as L
from ibis_b200 import params as prm

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def expected_header():
    return L.header_text().replace("#endif /* IBIS_LAYOUT_H */\n", prm.header_struct_text() + "\n#endif /* IBIS_LAYOUT_H */\n")


def test_layout_header_is_current():
    with open(os.path.join(REPO, "include", "ibis_layout.h")) as f:
        assert f.read() == expected_header()


def test_plane_counts():
    assert L.N_PROG == 71 and L.N_STAT == 135 and L.N_FORC == 12
    assert L.N_DIAG == 111 and L.N_ACC == 52
    assert L.leading_dim(1) == 32 and L.leading_dim(95333) % 32 == 0


def test_param_struct_size_matches_ctypes():
    import ctypes
    n_doubles = sum(n for _, n, _ in prm.PARAM_FIELDS)
    assert ctypes.sizeof(prm.IbisParamsC) == 8 * n_doubles + 8
