"""Writes tests/golden/reference_tests.json.

The problems and expected values are transcribed from the reference's own
solver tests (test/OptTests/*.jl in the CuClarabel tree); each entry cites the
file and lines it comes from.  The reference is Julia and cannot run in this
environment, so these deterministic test problems and their recorded answers
are the golden vectors that pin the CPU oracle.  Tests whose data comes from
Julia's MersenneTwister (basic_socp.jl, the SOCP cases) cannot be reproduced
without Julia and are not included.

Run:  python tests/golden/make_golden.py
"""
import json
import os

import numpy as np

Z, NN, SOC, EXP, POW, PSD = 0, 1, 2, 3, 4, 5


def dense(M):
    M = np.asarray(M, dtype=float)
    return M.tolist()


def case(name, src, P, q, A, b, cones, expect):
    return dict(name=name, source=src, P=dense(P), q=list(map(float, q)),
                A=dense(A), b=list(map(float, b)), cones=cones, expect=expect)


def basic_qp():
    # test/OptTests/basic_qp.jl:6-20
    P = [[4., 1], [1, 2]]
    c = [1., 1.]
    A = np.array([[1., 1], [1, 0], [0, 1]])
    l = np.array([1., 0, 0])
    u = np.array([1., 0.7, 0.7])
    A = np.vstack([-A, A])
    b = np.concatenate([-l, u])
    return P, c, A, b, [[NN, 3, 0], [NN, 3, 0]]


def basic_qp_dualinf():
    # test/OptTests/basic_qp.jl:23-33
    return [[1., 1], [1, 1]], [1., -1], [[1., 1], [1, 0]], [1., 1], [[NN, 2, 0]]


def basic_lp():
    # test/OptTests/basic_lp.jl:6-16
    A = np.vstack([np.eye(3), -np.eye(3)]) * 2
    return np.zeros((3, 3)), [3., -2, 1], A, np.ones(6), [[NN, 3, 0], [NN, 3, 0]]


def basic_exp():
    # test/OptTests/basic_exp.jl:6-37
    A1 = np.hstack([np.ones((1, 3)), np.zeros((1, 4))])
    A2 = np.hstack([np.zeros((3, 2)), -np.eye(3), np.zeros((3, 2))])
    A3 = np.zeros((3, 7))
    A3[0, 0] = -1
    A3[1, 2] = -1
    A3[2, 4] = -1
    A = np.vstack([A1, A2, A3])
    b = [10., 0, 0, 0, 0, 0, 0]
    c = [1.0, 0.5, -2., -0.1, 1.0, 3., 0.]
    P = np.eye(7) * 1e-1
    return P, c, A, b, [[Z, 1, 0], [NN, 3, 0], [EXP, 3, 0]]


def basic_pow():
    # test/OptTests/basic_pow.jl:6-38 (cone order: pow, pow, zero, zero)
    q = np.zeros(6)
    q[2] = q[5] = -1.
    A1 = np.eye(6)
    A2 = np.array([[1.0, 2.0, 0, 3.0, 0, 0]])
    A3 = np.array([[0, 0, 0, 0, 1.0, 0]])
    A = -np.vstack([A1, A2, A3])
    b = np.concatenate([np.zeros(6), [-3.], [-1.]])
    cones = [[POW, 3, 0.6], [POW, 3, 0.1], [Z, 1, 0], [Z, 1, 0]]
    return np.zeros((6, 6)), q, A, b, cones


def basic_sdp():
    # test/OptTests/basic_sdp.jl:6-17
    return (np.eye(6), np.zeros(6), np.eye(6), [-3., 1., 4., 1., 2., 5.],
            [[PSD, 3, 0]])


SDP_REF = [-3.0729833267361095, 0.3696004167288786, -0.022226685581313674,
           0.31441213129613066, -0.026739700851545107, -0.016084530571308823]


def main():
    out = []
    P, c, A, b, k = basic_qp()
    out.append(case("qp_feasible", "test/OptTests/basic_qp.jl:63-74", P, c, A, b, k,
                    dict(status="SOLVED", x=[0.3, 0.7], obj_val=1.8800000298331538,
                         obj_val_dual=1.8800000298331538, tol=1e-3)))
    b2 = b.copy()
    b2[0] = -1
    b2[3] = -1
    out.append(case("qp_primal_infeasible", "test/OptTests/basic_qp.jl:76-88",
                    P, c, A, b2, k, dict(status="PRIMAL_INFEASIBLE", obj_nan=True)))
    out.append(case("qp_univariate", "test/OptTests/basic_qp.jl:44-60",
                    [[1.]], [0.], [[1.]], [1.], [[NN, 1, 0]],
                    dict(x=[0.], obj_val=0.0, obj_val_dual=0.0, tol=1e-3)))
    P, c, A, b, k = basic_qp_dualinf()
    out.append(case("qp_dual_infeasible", "test/OptTests/basic_qp.jl:90-99",
                    P, c, A, b, k, dict(status="DUAL_INFEASIBLE", obj_nan=True)))
    out.append(case("qp_dual_infeasible_nonqsd", "test/OptTests/basic_qp.jl:101-114",
                    P, c, [A[0]], [b[0]], [[NN, 1, 0]],
                    dict(status="DUAL_INFEASIBLE", obj_nan=True)))
    P, c, A, b, k = basic_lp()
    out.append(case("lp_feasible", "test/OptTests/basic_lp.jl:26-36", P, c, A, b, k,
                    dict(status="SOLVED", x=[-0.5, 0.5, -0.5], obj_val=-3.0,
                         obj_val_dual=-3.0, tol=1e-3)))
    b2 = b.copy()
    b2[0] = -1
    b2[3] = -1
    out.append(case("lp_primal_infeasible", "test/OptTests/basic_lp.jl:38-50", P, c,
                    A, b2, k, dict(status="PRIMAL_INFEASIBLE", obj_nan=True)))
    A2 = A.copy()
    A2[3, 0] = 1.
    out.append(case("lp_dual_infeasible", "test/OptTests/basic_lp.jl:52-64", P,
                    [1., 0, 0], A2, b, k, dict(status="DUAL_INFEASIBLE", obj_nan=True)))
    A3 = A.copy()
    A3[0, 0] = np.finfo(float).eps
    A3[3, 0] = 0.0
    out.append(case("lp_dual_infeasible_illcond", "test/OptTests/basic_lp.jl:66-79",
                    P, [1., 0, 0], A3, b, k,
                    dict(status="DUAL_INFEASIBLE", obj_nan=True)))
    # test/OptTests/basic_eq_constrained.jl
    out.append(case("eq_constrained", "test/OptTests/basic_eq_constrained.jl:14-27",
                    np.eye(3), np.zeros(3), [[0., 1, 1], [0, 1, -1]], [2., 0],
                    [[Z, 2, 0]], dict(status="SOLVED", x=[0., 1., 1.], tol=1e-3)))
    out.append(case("eq_constrained_2", "test/OptTests/basic_eq_constrained.jl:29-42",
                    np.eye(3), [1., 2, 3], [[1., 1, 1], [0, 1, -1]], [2., 0],
                    [[Z, 2, 0]],
                    dict(status="SOLVED", x=[10 / 6, 1 / 6, 1 / 6], tol=1e-3)))
    Ar = [[0., 1, 1], [0, 1, -1], [0., 1, 1], [0, 1, -1]]
    out.append(case("eq_constrained_redundant",
                    "test/OptTests/basic_eq_constrained.jl:44-61", np.eye(3),
                    np.zeros(3), Ar, [2., 0, 2, 0], [[Z, 2, 0], [Z, 2, 0]],
                    dict(status="SOLVED", x=[0., 1., 1.], tol=1e-3)))
    out.append(case("eq_primal_infeasible",
                    "test/OptTests/basic_eq_constrained.jl:63-79", np.eye(3),
                    np.zeros(3),
                    [[0., 1, 1], [0, 1, -1], [1, 2, -1], [2, -1, 3]], np.ones(4),
                    [[Z, 4, 0]], dict(status="PRIMAL_INFEASIBLE")))
    Pd = np.eye(3)
    Pd[0, 0] = 0
    out.append(case("eq_dual_infeasible", "test/OptTests/basic_eq_constrained.jl:81-94",
                    Pd, np.ones(3), [[0., 1, 1], [0, 1, -1]], [2., 0], [[Z, 2, 0]],
                    dict(status="DUAL_INFEASIBLE")))
    # test/OptTests/basic_unconstrained.jl
    out.append(case("unconstrained", "test/OptTests/basic_unconstrained.jl:14-27",
                    np.eye(3), [1., 2, -3], np.zeros((0, 3)), [], [],
                    dict(status="SOLVED", x=[-1., -2., 3.], tol=1e-3)))
    out.append(case("unconstrained_dual_infeasible",
                    "test/OptTests/basic_unconstrained.jl:29-41", Pd, [1., 0, 0],
                    np.zeros((0, 3)), [], [], dict(status="DUAL_INFEASIBLE")))
    P, c, A, b, k = basic_exp()
    out.append(case("exp_feasible", "test/OptTests/basic_exp.jl:46-66", P, c, A, b, k,
                    dict(status="SOLVED",
                         x=[-9.425995201329599, 4.828561507482018, 14.59743362204262,
                            1.0000012112102774, 7.65314081561849, -29.99999978458479,
                            -0.0],
                         cost_primal=-54.41243965302268, tol=1e-3)))
    P, c, A, b, k = basic_pow()
    out.append(case("pow_feasible", "test/OptTests/basic_pow.jl:48-58", P, c, A, b, k,
                    dict(status="SOLVED", cost_primal=-1.8458, tol=1e-3)))
    P, c, A, b, k = basic_sdp()
    out.append(case("sdp_feasible", "test/OptTests/basic_sdp.jl:27-46", P, c, A, b, k,
                    dict(status="SOLVED", x=SDP_REF, obj_val=4.840076866013861,
                         tol=1e-3)))
    out.append(case("sdp_empty_cone", "test/OptTests/basic_sdp.jl:48-68", P, c, A, b,
                    k + [[PSD, 0, 0]],
                    dict(status="SOLVED", x=SDP_REF, obj_val=4.840076866013861,
                         tol=1e-3)))
    A2 = np.vstack([np.eye(6), -np.eye(6)])
    b2 = list(b) + [0.] * 6
    out.append(case("sdp_primal_infeasible", "test/OptTests/basic_sdp.jl:70-83",
                    P, c, A2, b2, k + k, dict(status="PRIMAL_INFEASIBLE")))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                        "reference_tests.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path, len(out), "cases")


if __name__ == "__main__":
    main()
