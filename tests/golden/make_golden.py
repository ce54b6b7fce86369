"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run in a checkout that has the reference sources (by default the reference
checkout beside this repository, override with REF_ROOT):
python tests/golden/make_golden.py

* The reference's runtime (cbits) is compiled in place with the GSL shim and
  the restated generated code (oracle/Makefile `ref`) and executed through
  oracle/oracle.py with kind "ref"; its outputs are the expected values.
* Model fixtures that the reference ships (examples/lda.py's d4_k4_v8 corpus)
  are read out of the reference's example file with `ast`, not retyped.
The fixtures are small .npz files; the tests read only these files, never the
reference.
"""
import ast
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF_ROOT = os.environ.get("REF_ROOT", os.path.join(os.path.dirname(ROOT), "reference"))

from oracle import oracle as O  # noqa: E402


def example_arrays(path, func_name):
    """Literal np.array(...) assignments inside one function of a reference
    example script, evaluated without running the script.  The examples are
    Python 2, so `print x` statement lines are dropped before parsing."""
    lines = [ln for ln in open(path).read().splitlines()
             if not ln.strip().startswith(("print ", "get_ipython"))]
    tree = ast.parse("\n".join(lines))
    out = {}
    for node in ast.walk(tree):
        if isinstance(node, ast.FunctionDef) and node.name == func_name:
            for st in node.body:
                if (isinstance(st, ast.Assign) and len(st.targets) == 1
                        and isinstance(st.targets[0], ast.Name) and isinstance(st.value, ast.Call)
                        and getattr(st.value.func, "attr", "") == "array" and st.value.args
                        and isinstance(st.value.args[0], ast.List)):
                    try:
                        out[st.targets[0].id] = ast.literal_eval(st.value.args[0])
                    except ValueError:
                        pass
    return out


def example_values(path, func_name, names):
    """Values of simple assignments (`mu = [np.array([...]), ...]`,
    `covs = np.matrix([...])`) inside one function of a reference example."""
    lines = [ln for ln in open(path).read().splitlines()
             if not ln.strip().startswith(("print ", "get_ipython"))]
    tree = ast.parse("\n".join(lines))

    def ev(node):
        if isinstance(node, ast.Call) and getattr(node.func, "attr", "") in ("array", "matrix"):
            return np.array(ast.literal_eval(node.args[0]), dtype=np.float64)
        if isinstance(node, ast.List):
            return [ev(e) for e in node.elts]
        return ast.literal_eval(node)

    out = {}
    for node in ast.walk(tree):
        if isinstance(node, ast.FunctionDef) and node.name == func_name:
            for st in ast.walk(node):
                if isinstance(st, ast.Assign):
                    for tgt in st.targets:
                        if isinstance(tgt, ast.Name) and tgt.id in names:
                            try:
                                out[tgt.id] = ev(st.value)
                            except (ValueError, TypeError, AttributeError, IndexError):
                                pass
    return out


def lda_fixture_d4_k4_v8():
    arrs = example_arrays(os.path.join(REF_ROOT, "examples", "lda.py"), "mk_synthetic_dataset_d4_k4_v8")
    docs = [np.array(arrs[k], np.int32) for k in ("w1", "w2", "w3", "w4")]
    N = np.array(arrs["N"], np.int32)
    assert [len(d) for d in docs] == list(N)
    return docs


def make_primitives(ref):
    shapes = np.array([0.01, 0.05, 0.1, 0.5, 0.99, 1.0, 1.01, 2.5, 3.7, 10.0, 50.0, 200.5])
    gam = np.array([[ref.gamma_sample(s, r, 11, e, 3, O.TAG_PHI) for e in range(8)]
                    for s, r in [(s, 1.0) for s in shapes] + [(2.0, 0.5), (0.3, 4.0)]])
    rng = np.random.default_rng(5)
    pmfs = rng.random((64, 7)) ** 3
    pmfs[3, :] = 0.0
    pmfs[3, 4] = 1.0
    disc = np.array([ref.unnorm_disc_samp(p, 19, i, 2, O.TAG_Z) for i, p in enumerate(pmfs)], np.int32)
    np.savez_compressed(os.path.join(HERE, "primitives.npz"), shapes=shapes, gamma=gam,
                        pmfs=pmfs, disc=disc)


def make_lda(ref):
    # (1) the reference's own example corpus, 10 sweeps from the uniform init
    docs = lda_fixture_d4_k4_v8()
    D, K, V = 4, 4, 8
    off = np.concatenate([[0], np.cumsum([len(d) for d in docs])]).astype(np.int32)
    w = np.concatenate(docs).astype(np.int32)
    alpha, beta = np.full(K, 0.1), np.full(V, 0.01)
    theta, phi = np.full((D, K), 1.0 / K), np.full((K, V), 1.0 / V)
    z = np.zeros(len(w), np.int32)
    thetas, phis, zs = [], [], []
    for s in range(10):
        ref.lda_sweeps(off, w, alpha, beta, theta, phi, z, 0, s, 1)
        thetas.append(theta.copy()); phis.append(phi.copy()); zs.append(z.copy())
    np.savez_compressed(os.path.join(HERE, "lda_d4_k4_v8.npz"), doc_off=off, w=w, alpha=alpha,
                        beta=beta, theta=np.array(thetas), phi=np.array(phis), z=np.array(zs))

    # (2) a synthetic corpus of the benchmark's shape family, reduced size
    from augurv2_b200.lda import synthetic_corpus
    K, V, D = 12, 300, 40
    off, w = synthetic_corpus(K, V, D, 60, 0.1, 0.01, seed=3)
    alpha, beta = np.full(K, 0.1), np.full(V, 0.01)
    rng = np.random.default_rng(4)
    theta = rng.dirichlet(np.full(K, 0.5), size=D)
    phi = rng.dirichlet(np.full(V, 0.1), size=K)
    z = rng.integers(0, K, size=len(w)).astype(np.int32)
    theta0, phi0, z0 = theta.copy(), phi.copy(), z.copy()
    ref.lda_sweeps(off, w, alpha, beta, theta, phi, z, 7, 0, 3)
    np.savez_compressed(os.path.join(HERE, "lda_k12_v300_d40.npz"), doc_off=off, w=w, alpha=alpha,
                        beta=beta, theta0=theta0, phi0=phi0, z0=z0, theta=theta, phi=phi, z=z)


def make_hlr(ref):
    """HLR on the reference's hlr.rv model (Exponential variance prior with
    bias) and on the InvGamma variant without bias: log-densities, gradients
    and HMC / NUTS / MWG / reflective-slice transitions of the reference's
    own kernels."""
    out = {}
    for name, (N, D, has_b, vprior) in {"hlr": (120, 6, True, "exponential"),
                                        "ighlr": (150, 4, False, "invgamma")}.items():
        X, y, beta, s2 = O.hlr_synthetic(N, D, seed=N + D, has_b=has_b)
        m = O.HlrModel(X, y, has_b=has_b, vprior=vprior, lam=1.0, a0=1.0, s0=1.0, compat=True)
        rng = np.random.default_rng(N)
        par0 = np.concatenate([beta * 0.7, [0.2 if has_b else 0.0], [max(0.3, s2)]])
        blocks = {"theta": list(range(D)), "v": [D + 1], "joint": [D + 1] + ([D] if has_b else []) + list(range(D))}
        if has_b:
            blocks["b"] = [D]
        pars = par0 + 0.1 * rng.standard_normal((5, D + 2))
        pars[:, D + 1] = np.abs(pars[:, D + 1]) + 0.1
        if not has_b:
            pars[:, D] = 0.0
        rec = {"X": X, "y": y, "pars": pars, "N": N, "D": D, "has_b": int(has_b), "vprior": m.vprior}
        for bname, idx in blocks.items():
            rec["ll_" + bname] = np.array([O.hlr_ll(ref, m, p, idx) for p in pars])
            rec["grad_" + bname] = np.array([O.hlr_grad(ref, m, p, idx) for p in pars])
            rec["idx_" + bname] = np.array(idx, np.int32)
        # chains of transitions (seed 7): HMC on theta, NUTS on the joint block, MWG on v
        p = par0.copy(); hmc = []
        for it in range(6):
            O.hlr_hmc(ref, m, p, blocks["theta"], 0.3, 0.05, 7, it)
            hmc.append(p.copy())
        p = par0.copy(); nuts = []
        for it in range(6):
            O.hlr_nuts(ref, m, p, blocks["joint"], 0.05, 7, it)
            nuts.append(p.copy())
        p = par0.copy(); mwg = []
        for it in range(6):
            O.hlr_mwg(ref, m, p, D + 1, 0.5, 7, it)
            mwg.append(p.copy())
        p = par0.copy(); rslice = []
        for it in range(8):
            O.hlr_rslice(ref, m, p, blocks["theta"], 0.5, 0.05, 7, it)
            rslice.append(p.copy())
        rec.update(par0=par0, hmc=np.array(hmc), nuts=np.array(nuts), mwg=np.array(mwg), rslice=np.array(rslice))
        np.savez_compressed(os.path.join(HERE, name + "_golden.npz"), **rec)


def make_gmm(ref):
    """mvgmm with the centres and covariance of the reference's example
    (examples/mvgmm.py mk_synthetic_dataset_k3_d2; points drawn here with a
    seed), and an hmvgmm instance of the benchmark's construction."""
    vals = example_values(os.path.join(REF_ROOT, "examples", "mvgmm.py"), "mk_synthetic_dataset_k3_d2",
                          {"mu", "covs"})
    centres, covs = np.array(vals["mu"]), np.array(vals["covs"])
    K, d, N = centres.shape[0], centres.shape[1], 60
    rng = np.random.default_rng(60)
    Lc = np.linalg.cholesky(covs)
    Y = np.array([centres[n % K] + Lc @ rng.standard_normal(d) for n in range(N)])
    Y = Y.astype(np.float32).astype(np.float64)
    mu0, cov0 = np.zeros(d), np.eye(d)
    pis = np.full(K, 1.0 / K)
    g = O.GmmModel(Y, K, mu0, cov0, True)
    mu, z = np.zeros((K, d)), np.zeros(N, np.int32)
    mus, zs = [], []
    for it in range(8):
        O.gmm_sweep(ref, g, pis, mu, covs, z, 1, it)
        mus.append(mu.copy()); zs.append(z.copy())
    es = O.gmm_eslice(ref, g, mus[-1], covs, zs[-1], 2, 0)
    mw = O.gmm_mwg(ref, g, mus[-1], covs, zs[-1], cov0, 2, 0)
    np.savez_compressed(os.path.join(HERE, "mvgmm_k3_d2.npz"), Y=Y, covs=covs, pis=pis, mu0=mu0, cov0=cov0,
                        mu=np.array(mus), z=np.array(zs), eslice=es, mwg=mw)

    K, d, N = 4, 5, 400
    Y, z0, mus_t, covs_t, pis_t = O.gmm_synthetic(N, K, d, seed=7)
    g = O.GmmModel(Y, K, np.zeros(d), 25 * np.eye(d), False, alpha=np.ones(K), df=d + 2, scale0=np.eye(d))
    pis, mu, cov, z = pis_t.copy(), mus_t.copy(), covs_t.copy(), z0.copy()
    rec = dict(Y=Y, mu_init=mus_t, cov_init=covs_t, pis_init=pis_t, z_init=z0)
    P, M, Cv, Z = [], [], [], []
    for it in range(4):
        O.gmm_sweep(ref, g, pis, mu, cov, z, 3, it)
        P.append(pis.copy()); M.append(mu.copy()); Cv.append(cov.copy()); Z.append(z.copy())
    rec.update(pis=np.array(P), mu=np.array(M), cov=np.array(Cv), z=np.array(Z))
    np.savez_compressed(os.path.join(HERE, "hmvgmm_k4_d5.npz"), **rec)


CONJ_KINDS = ["beta_bernoulli", "beta_geometric", "gamma_poisson", "gamma_exponential",
              "gamma_gammashape", "gamma_invgamma", "normal_normalmean"]


def conj_inputs(kind, seed):
    """Ragged groups (some empty) of observations of the kind's likelihood,
    and its hyper-parameters (per group for odd kinds, shared otherwise)."""
    rng = np.random.default_rng(seed)
    G = 37
    lens = rng.integers(0, 60, G)
    lens[[3, 17]] = 0
    off = np.zeros(G + 1, np.int32)
    np.cumsum(lens, out=off[1:])
    n = int(off[-1])
    x = {"beta_bernoulli": lambda: (rng.random(n) < 0.3).astype(np.float64),
         "beta_geometric": lambda: rng.geometric(0.4, n).astype(np.float64) - 1.0,
         "gamma_poisson": lambda: rng.poisson(3.0, n).astype(np.float64),
         "gamma_exponential": lambda: rng.exponential(0.5, n),
         "gamma_gammashape": lambda: rng.gamma(2.0, 0.25, n),
         "gamma_invgamma": lambda: 1.0 / rng.gamma(3.0, 1.0 / 2.0, n),
         "normal_normalmean": lambda: rng.normal(1.5, 2.0, n)}[kind]()
    aux = rng.uniform(0.5, 4.0, n) if kind in ("gamma_gammashape", "gamma_invgamma") else None
    k = CONJ_KINDS.index(kind)
    if k % 2:
        h0, h1 = rng.uniform(0.05, 3.0, G), rng.uniform(0.05, 3.0, G)
        h2 = rng.uniform(0.5, 5.0, G)
    else:
        h0, h1, h2 = 0.7, 1.3, 4.0
    if kind == "normal_normalmean" and np.ndim(h0) == 0:
        h0 = -0.5
    return off, x, aux, h0, h1, h2


def make_conj(ref):
    rec = {}
    for k, kind in enumerate(CONJ_KINDS):
        off, x, aux, h0, h1, h2 = conj_inputs(kind, 100 + k)
        for it in (0, 5):
            out, ssum, saux = ref.conj_scalar(k, off, x, h0, h1, h2, aux=aux, seed=23, it=it)
            rec["%s_it%d_out" % (kind, it)] = out
            rec["%s_it%d_sum" % (kind, it)] = ssum
            rec["%s_it%d_aux" % (kind, it)] = saux
    np.savez_compressed(os.path.join(HERE, "conj_scalar.npz"), **rec)


def make_models():
    """The reference's model files (compiler/augur/test/*.rv) and the model
    strings and schedules of its examples, as parser fixtures."""
    import json
    out = {"rv": {}, "examples": {}}
    tdir = os.path.join(REF_ROOT, "compiler", "augur", "test")
    for f in sorted(os.listdir(tdir)):
        if f.endswith(".rv"):
            out["rv"][f[:-3]] = open(os.path.join(tdir, f)).read()
    for ex in ("hlr", "lda", "mvgmm"):
        lines = [ln for ln in open(os.path.join(REF_ROOT, "examples", ex + ".py")).read().splitlines()
                 if not ln.strip().startswith(("print ", "get_ipython"))]
        tree = ast.parse("\n".join(lines))
        rec = {"scheds": []}
        for node in tree.body:
            if isinstance(node, ast.Assign) and isinstance(node.targets[0], ast.Name) \
                    and isinstance(node.value, ast.Constant) and isinstance(node.value.value, str):
                name = node.targets[0].id
                if name.startswith("augur_"):
                    rec["model"] = node.value.value
                elif name.startswith("sched"):
                    rec["scheds"].append(node.value.value)
        out["examples"][ex] = rec
    with open(os.path.join(HERE, "models.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    make_models()
    O.build_oracle()
    ref = O.Oracle("ref")
    make_primitives(ref)
    make_lda(ref)
    make_hlr(ref)
    make_gmm(ref)
    make_conj(ref)
    print("golden fixtures written to", HERE)
