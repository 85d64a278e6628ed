"""Generate the anisotropic-law fixtures by running the REFERENCE's own symbolic derivation
(doc/anisotropic.py) and evaluating its expressions in FP64 on seeded inputs.

    python tests/golden/make_aniso_golden.py <reference checkout>   (or JAXMATERIALS_REF in the environment)

The reference module builds, with sympy, the stress law sigma = C : eps over the 21
independent stiffness entries (stress_strain, :20-42), the acoustic matrix
K_ki = C^0_kjil xi_j xi_l (acoustic_matrix, :46-95) and the Green operator
Gamma^0_klij = 1/4 (N xi xi, symmetrised) with N = K^-1 (fourier_solve, :98-128), and
writes them as LaTeX. It is imported unchanged (from a temporary working directory, where
its module-level code writes its .tex files); its module-level name `latex`, through which
every final expression passes, is replaced by a recorder, so the very sympy expressions it
prints are captured and evaluated here (sympy.lambdify, FP64).

Writes tests/golden/reference_aniso.npz:
  c21 (S, 21), eps (S, 6)          -> sigma (S, 6)
  c0 (S, 21), xi (S, 3) unit       -> K (S, 3, 3) (symmetric; the lower triangle is the
                                      reference's), N = K^-1 (S, 3, 3)
                                   -> gamma (S, 6, 6) symmetric, gamma[a, b] = Gamma^0 of
                                      Voigt pairs a = (k, l), b = (i, j)
"""

import importlib.util
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference_module(ref):
    path = os.path.join(ref, "doc", "anisotropic.py")
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)
        try:
            spec = importlib.util.spec_from_file_location("reference_anisotropic", path)
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
        finally:
            os.chdir(cwd)
    return mod


def capture(mod, fn, *args, **kw):
    """Run one of the module's printers and return the expressions it passed to latex()."""
    seen = []
    original = mod.latex

    def recorder(expr, *a, **k):
        seen.append(expr)
        return original(expr, *a, **k)

    mod.latex = recorder
    try:
        fn(*args, **kw)
    finally:
        mod.latex = original
    return seen


def plain_symbols(exprs, sp):
    """Replace the array elements C[k], varepsilon[b], C^0[k] by plain symbols; returns the
    rewritten expressions and the symbol lookup by (array name, index)."""
    table = {}
    out = []
    for e in exprs:
        repl = {}
        for el in e.atoms(sp.tensor.array.expressions.ArrayElement):
            name = str(el.name)
            idx = int(el.indices[0])
            key = (name, idx)
            if key not in table:
                table[key] = sp.Symbol(f"{name.replace('^', '').replace('{', '').replace('}', '')}_{idx}")
            repl[el] = table[key]
        out.append(e.xreplace(repl))
    return out, table


def main(ref):
    import sympy as sp

    mod = load_reference_module(ref)
    vi, ci = mod.voigt_indices, mod.C_indices
    rng = np.random.default_rng(20240611)
    S = 24

    # ---- stress law
    sig_exprs, table = plain_symbols(capture(mod, mod.stress_strain, vi, ci), sp)
    c_syms = [table[("C", k)] for k in range(21)]
    e_syms = [table[("varepsilon", b)] for b in range(6)]
    f_sig = sp.lambdify(c_syms + e_syms, sig_exprs, "numpy")
    c21 = rng.normal(size=(S, 21))
    c21[:, :6] += 8.0  # a diagonally dominant (positive definite) stiffness
    eps = rng.normal(size=(S, 6))
    sigma = np.array([f_sig(*c21[s], *eps[s]) for s in range(S)], dtype=np.float64)

    # ---- acoustic matrix (lower triangle K_ij, j <= i, in the order printed)
    k_exprs = capture(mod, mod.acoustic_matrix, vi, ci, isotropic=False)
    k_exprs, table = plain_symbols(k_exprs, sp)
    xi_syms = sorted({s for e in k_exprs for s in e.free_symbols if "xi" in str(s)}, key=str)
    c0_syms = [table[("C^{0}", k)] for k in range(21)]
    f_k = sp.lambdify(c0_syms + xi_syms, k_exprs, "numpy")
    c0 = rng.normal(size=(S, 21)) * 0.3
    c0[:, :6] += 5.0
    xi = rng.normal(size=(S, 3))
    xi /= np.linalg.norm(xi, axis=1, keepdims=True)
    kmat = np.zeros((S, 3, 3))
    pos = [(i, j) for i in range(3) for j in range(i + 1)]
    for s in range(S):
        vals = f_k(*c0[s], *xi[s])
        for (i, j), v in zip(pos, vals):
            kmat[s, i, j] = kmat[s, j, i] = float(v)
    nmat = np.linalg.inv(kmat)

    # ---- Green operator (upper triangle a <= b, in the order printed)
    g_exprs = capture(mod, mod.fourier_solve, vi)
    n_names = ["N^{0}_{00}", "N^{0}_{01}", "N^{0}_{02}", "N^{0}_{11}", "N^{0}_{12}", "N^{0}_{22}"]
    n_syms = [sp.Symbol(n) for n in n_names]
    gxi = sorted({s for e in g_exprs for s in e.free_symbols if "xi" in str(s)}, key=str)
    f_g = sp.lambdify(n_syms + gxi, g_exprs, "numpy")
    gamma = np.zeros((S, 6, 6))
    upper = [(a, b) for a in range(6) for b in range(a, 6)]
    for s in range(S):
        n6 = [nmat[s, 0, 0], nmat[s, 0, 1], nmat[s, 0, 2], nmat[s, 1, 1], nmat[s, 1, 2], nmat[s, 2, 2]]
        vals = f_g(*n6, *xi[s])
        for (a, b), v in zip(upper, vals):
            gamma[s, a, b] = gamma[s, b, a] = float(v)

    out = os.path.join(HERE, "reference_aniso.npz")
    np.savez_compressed(out, c21=c21, eps=eps, sigma=sigma, c0=c0, xi=xi, K=kmat, N=nmat,
                        gamma=gamma)
    print("wrote", out, "samples", S)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["JAXMATERIALS_REF"])
