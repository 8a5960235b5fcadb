"""test/UnitTests/test_json.jl on this solver: write, read back, solve both."""
import numpy as np
import pytest
import scipy.sparse as sp

from cuclarabel_b200 import (NonnegativeConeT, Settings, Solver, SolverStatus, ZeroConeT,
                             read_from_file, write_to_file)

pytestmark = pytest.mark.gpu


def test_json_round_trip_solves_the_same(cuda_device, tmp_path):
    P = sp.csc_matrix(np.array([[4.0, 1.0], [1.0, 2.0]]))
    c = np.array([1.0, 1.0])
    A = sp.csc_matrix(np.array([[1.0, 1.0], [1.0, 0.0], [0.0, 1.0]]))
    b = np.array([1.0, 1.0, 1.0])
    cones = [NonnegativeConeT(1), ZeroConeT(1), NonnegativeConeT(1)]
    solver = Solver(P, c, A, b, cones)
    f = str(tmp_path / "problem.json")
    write_to_file(solver, f)
    solver2 = read_from_file(f)
    s1, s2 = solver.solve(), solver2.solve()
    assert np.allclose(s1.x, s2.x, atol=1e-10)
    assert s1.status == s2.status
    solver3 = read_from_file(f, Settings(max_iter=1))
    assert solver3.solve().status == SolverStatus.MAX_ITERATIONS


def test_written_file_tracks_data_updates(cuda_device, tmp_path):
    P = sp.csc_matrix(np.array([[4.0, 1.0], [1.0, 2.0]]))
    A = sp.csc_matrix(np.array([[1.0, 1.0], [1.0, 0.0], [0.0, 1.0]]))
    cones = [NonnegativeConeT(1), ZeroConeT(1), NonnegativeConeT(1)]
    solver = Solver(P, np.array([1.0, 1.0]), A, np.array([1.0, 1.0, 1.0]), cones)
    solver.update_q(np.array([2.0, -1.0]))
    solver.update_b(np.array([1.5, 1.0, 2.0]))
    f = str(tmp_path / "updated.json")
    write_to_file(solver, f)
    s1, s2 = solver.solve(), read_from_file(f).solve()
    assert s1.status == s2.status == SolverStatus.SOLVED
    assert np.allclose(s1.x, s2.x, atol=1e-9)
