"""State text I/O against the reference's own (src/model.cpp:254-383,636-638,
src/common.cpp:161-181): files written by the drop-in State equal the
reference's byte for byte, and files written by the reference load into the
same tile (periodic halos filled from the opposite side)."""
import numpy as np
import pytest

import tsref

pytestmark = pytest.mark.skipif(not tsref.available(), reason="compiled reference not built")

# (dim_x, L, dim_y, periodic_x, periodic_y, one_d)
LATTICES = [(20, 4.0, 16, False, False, False), (16, 4.0, 12, True, True, False),
            (18, 4.0, 14, True, False, False), (24, 6.0, 0, False, False, True)]


def _pair(case, seed):
    import trottersuzuki_b200 as ts
    nx, L, ny, px, py, one_d = case
    if one_d:
        grid = ts.Lattice1D(nx, L, px)
        cfg = tsref.make_config(nx, L, 0, None, px, False)
    else:
        grid = ts.Lattice2D(nx, L, ny, L, px, py)
        cfg = tsref.make_config(nx, L, ny, L, px, py)
    rng = np.random.default_rng(seed)
    shape = (grid.dim_y, grid.dim_x)
    psi = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    psi[0, 0] = -0.0 + 1e-300j  # formatting corner cases
    st = ts.State(grid)
    st.init_state_matrix(psi.real, psi.imag)
    return grid, st, cfg, psi


@pytest.mark.parametrize("case", LATTICES, ids=["closed", "periodic", "periodic_x", "1d"])
def test_written_files_equal_the_reference(case, tmp_path):
    grid, st, cfg, psi = _pair(case, 1)
    for kind, write in ((0, st.write_to_file), (1, st.write_particle_density),
                        (2, st.write_phase)):
        ours, ref = tmp_path / f"ours{kind}", tmp_path / f"ref{kind}"
        write(str(ours))
        tsref.write_state(cfg, psi, kind, str(ref))
        suffix = {0: "", 1: "-density", 2: "-phase"}[kind]
        a = (tmp_path / (f"ours{kind}" + suffix)).read_bytes()
        b = (tmp_path / (f"ref{kind}" + suffix)).read_bytes()
        assert a == b, kind


@pytest.mark.parametrize("case", LATTICES, ids=["closed", "periodic", "periodic_x", "1d"])
def test_reference_files_load_into_the_same_tile(case, tmp_path):
    grid, st, cfg, psi = _pair(case, 2)
    f = tmp_path / "state"
    tsref.write_state(cfg, psi, 0, str(f))
    want = tsref.load_state(cfg, str(f))
    import trottersuzuki_b200 as ts
    st2 = ts.State(grid)
    st2.loadtxt(str(f))
    got = st2.get_state()
    # the reference's loader leaves cells it does not cover at their previous
    # value (zero in a fresh State), as here
    assert np.array_equal(got, want)
