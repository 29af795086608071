"""Known-answer cases of the sift, stated explicitly.  The expected values are
what the reference kernel itself produced for these inputs (recorded in the
golden fixtures), and the cases are the ones its documentation and bug
history describe: an all-zero warm-up trace, a pure tone, a linear trend, a
trace with more than max_extrema extrema per side, the iteration cap, a
one-sample trace.  The CPU oracle must give them (always); the B200 path must
give them too (GPU)."""
import numpy as np
import pytest

from oracle import emd_oracle as O

import cases


def _case(name):
    g = {c["name"]: c for c in cases.groups()}[name]
    cfg = O.OracleConfig(**g["cfg"])
    return g["signals"], g["T"], cfg


def _known(run):
    """run(X, T, cfg) -> (imfs [B, mi, N], n_imfs, overflow, debug_n) for each case."""
    # all-zero warm-up trace: no IMF, no sift pass, no residue row
    X, T, cfg = _case("warmup64")
    imfs, n, ovf, dn = run(X, T, cfg)
    assert n[0] == 0 and ovf[0] == 0 and (dn[0] == -1).all() and not imfs[0].any()
    # edge512 rows: pure tone, linear trend
    X, T, cfg = _case("edge512")
    imfs, n, ovf, dn = run(X[:2], T, cfg)
    # a pure tone is one IMF after a single sift pass; the ~zero residue is dropped
    assert n[0] == 1 and ovf[0] == 0 and dn[0][0] == 1 and (dn[0][1:] == -1).all()
    np.testing.assert_allclose(imfs[0][0], X[0], atol=1e-9)
    assert not imfs[0][1:].any()
    # a linear trend has no IMF: one row, the residue, equal to the input, no sift
    assert n[1] == 1 and ovf[1] == 0 and (dn[1] == -1).all()
    assert np.array_equal(imfs[1][0], X[1]) and not imfs[1][1:].any()
    # a chirp with more than max_extrema extrema per side: overflow, and its
    # first IMF runs into the iteration cap (debug_n logs the cap)
    X, T, cfg = _case("chirp6000")
    imfs, n, ovf, dn = run(X, T, cfg)
    assert ovf[0] == 1 and dn[0][0] == cfg.max_iteration
    # the iteration cap of a small config: every overflowed trace logs it
    X, T, cfg = _case("small_cfg")
    imfs, n, ovf, dn = run(X, T, cfg)
    capped = (dn == cfg.max_iteration).any(axis=1)
    assert (ovf.astype(bool) == capped).all() and capped.sum() >= 6
    # a one-sample trace: no sift, the residue row is the sample
    X, T, cfg = _case("tiny1")
    imfs, n, ovf, dn = run(X, T, cfg)
    assert n[0] == 1 and imfs[0][0][0] == X[0][0] and (dn[0] == -1).all()


def test_known_answers_oracle(golden):
    def run(X, T, cfg):
        rs = [O.emd_signal(x, T, cfg) for x in X]
        return (np.stack([r.imfs for r in rs]), np.array([r.n_imfs for r in rs]),
                np.array([r.overflow for r in rs]).astype(int), np.stack([r.debug_n for r in rs]))
    _known(run)
    # and these are the reference kernel's own recorded answers
    for name in ("warmup64", "edge512", "chirp6000", "small_cfg", "tiny1"):
        X, T, cfg = _case(name)
        rs = [O.emd_signal(x, T, cfg) for x in X]
        assert [r.n_imfs for r in rs] == golden[f"{name}__nofma__n_imfs"].tolist()


@pytest.mark.gpu
def test_known_answers_b200():
    import torch
    from cuda_emd import EMDKernelConfig

    def run(X, T, cfg):
        c = EMDKernelConfig(max_extrema=cfg.max_extrema, nbsym=cfg.nbsym,
                            max_iteration=cfg.max_iteration, max_imfs=cfg.max_imfs,
                            threads_per_block=cfg.threads_per_block)
        L = c.build()
        out = L.run(torch.from_numpy(np.ascontiguousarray(X)).cuda(),
                    torch.from_numpy(np.ascontiguousarray(T)).cuda())
        L.check_status()
        imfs, n, ovf, dn, de, dz = (o.cpu().numpy() for o in out)
        return imfs, n, ovf, dn
    _known(run)
