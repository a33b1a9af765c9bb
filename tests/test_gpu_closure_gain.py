"""What the learned closure gains over the solver without it, on a short
small-grid run: hold-energy forced DNS at 64^3 (nu = 4e-3) filtered to 32^3
(k_c = 10); the closure is fitted a priori on the filtered DNS stresses, then
tuned a posteriori through the discrete adjoint of the LES (windows of 48
steps, the squared log-error of the LES spectrum against the filtered DNS);
each LES runs 1200 steps from the first filtered snapshot.  The classical
Chollet-Lesieur spectral eddy viscosity runs beside them.  The maximum
relative E(k) error over k <= k_c must fall from the unmodelled solver to
the a-priori closure and again to the a-posteriori one."""

import importlib

import pytest

pytestmark = pytest.mark.gpu

les = importlib.import_module("3dhit_b200.les")


def test_closure_beats_the_unmodelled_solver_and_adjoint_tuning_improves_it():
    data = les.make_dataset(fine_n=64, coarse_n=32, nu=4e-3, spinup=800, snapshots=40, every=25)
    model, _ = les.train(data, steps=200, batch_snapshots=8, val_snapshots=4)
    ref = data["spectra"].mean(0)

    def err(m):
        r = les.run_les(data, m, steps=1200, sample_every=20, discard=200)
        assert r["finite"]
        rel = (r["spectrum"] / ref - 1).abs()
        return float(rel.max()), float(rel.mean())

    none = err(None)
    prior = err(model)
    cls = les.run_spectral_eddy_viscosity_les(data, 1200, 200, sample_every=20)
    cls_err = float((cls / ref - 1).abs().max())
    hist = les.train_a_posteriori(data, model, iters=30, window=48, lr=3e-4)
    post = err(model)
    print(f"max / mean |E_LES/E_DNS - 1|, k <= 10: no closure {none}, Chollet-Lesieur {cls_err:.3f}, "
          f"a priori {prior}, a posteriori {post}; "
          f"a-posteriori loss {hist[0][2]:.3f} -> {hist[-1][2]:.3f}")
    assert prior[0] < none[0]
    assert cls_err < none[0]  # the classical closure removes the unmodelled solver's cut-off pile-up too
    assert post[0] < prior[0] and post[1] < prior[1]


def test_a_posteriori_model_selection_keeps_the_best_scored_weights():
    """With ``select_every`` the tuning scores the weights by a held-out LES
    (before the first iteration, every few iterations and after the last)
    and ends on the best-scored ones.  The LES is deterministic, so scoring
    the final weights again reproduces the lowest recorded score exactly."""
    data = les.make_dataset(fine_n=64, coarse_n=32, nu=4e-3, spinup=400, snapshots=12, every=25)
    model, _ = les.train(data, steps=60, batch_snapshots=4, val_snapshots=2)
    les.train_a_posteriori(data, model, iters=8, window=24, lr=3e-4, select_every=4, select_steps=400)
    sel = model.a_posteriori_selection
    assert [it for it, _ in sel] == [0, 4, 8]
    ref = data["spectra"].mean(0)
    r = les.run_les(dict(data, u0_coarse=data["U"][-1]), model, steps=400, sample_every=50, discard=80)
    assert r["finite"]
    again = float((r["spectrum"] / ref - 1).abs().max())
    assert again == min(sc for _, sc in sel), (again, sel)
