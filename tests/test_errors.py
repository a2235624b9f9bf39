"""Argument validation of the learned-form, batched-replica and Ewald entry points: every bad call
returns PD_EINVAL with a message before touching the device (runs without a GPU)."""
import ctypes as C

import pytest


def _lib(pd):
    return pd._native.lib()


def _expect_einval(pd, name, *args):
    L = _lib(pd)
    code = getattr(L, name)(*args)
    assert code == pd._native.PD_EINVAL, (name, code)
    assert L.pd_last_error().decode()


def test_network_entry_points_reject_null_handles(pd):
    _expect_einval(pd, "pd_mlp_forward", None, 0, 4, 0, 0, 0, None)
    _expect_einval(pd, "pd_mlp_train", None, 0, 0, 4, C.c_float(1.0), None)
    _expect_einval(pd, "pd_mlp_adam", None, C.c_float(1e-3), C.c_float(0.9), C.c_float(0.999), C.c_float(1e-8),
                   C.c_float(1.0), None)
    _expect_einval(pd, "pd_mlp_set_params", None, None)
    _expect_einval(pd, "pd_mlp_create", None)
    assert _lib(pd).pd_mlp_param_count() == pd.learned.PARAM_COUNT


@pytest.mark.parametrize("field,value", [("nb", 0), ("nb", 9), ("sigma", 0.0), ("tau", -1.0), ("cap", 0),
                                         ("rcut", 0.0)])
def test_learned_create_validates(pd, field, value):
    p = pd._native.LearnedParams()
    for k, v in dict(rcut=6.0, skin=1.0, cap=64, mu0=0.5, dmu=0.35, sigma=0.35, nb=8, nu0=2.0, dnu=0.5,
                     tau=0.45).items():
        setattr(p, k, v)
    setattr(p, field, value)
    h = C.c_void_p()
    _expect_einval(pd, "pd_learned_create", C.byref(h), C.byref(p), 100, pd._native.dbl3((20.0, 20.0, 20.0)))
    _expect_einval(pd, "pd_learned_create", C.byref(h), C.byref(pd._native.LearnedParams()), 0,
                   pd._native.dbl3((20.0, 20.0, 20.0)))


def test_batch_create_validates(pd):
    N = pd._native
    good = pd.batch.replica_params("lj", (10.0, 10.0, 10.0), 500)
    reps = (N.BatchReplica * 1)(good)
    h = C.c_void_p()
    _expect_einval(pd, "pd_batch_create", C.byref(h), reps, 1, C.c_float(0.3), 64, 3)        # lanes
    _expect_einval(pd, "pd_batch_create", C.byref(h), reps, 1, C.c_float(-0.1), 64, 4)       # skin
    _expect_einval(pd, "pd_batch_create", C.byref(h), reps, 1, C.c_float(0.3), 0, 4)         # capacity
    _expect_einval(pd, "pd_batch_create", C.byref(h), reps, 0, C.c_float(0.3), 64, 4)        # no replicas
    small = (N.BatchReplica * 1)(pd.batch.replica_params("lj", (5.0, 10.0, 10.0), 100))
    _expect_einval(pd, "pd_batch_create", C.byref(h), small, 1, C.c_float(0.3), 64, 4)       # box < 2 r_list
    empty = (N.BatchReplica * 1)(pd.batch.replica_params("wca", (10.0, 10.0, 10.0), 0))
    _expect_einval(pd, "pd_batch_create", C.byref(h), empty, 1, C.c_float(0.3), 64, 4)       # empty replica
    with pytest.raises(ValueError):
        pd.batch.replica_params("coulomb", (10.0, 10.0, 10.0), 10)


def test_ewald_oracle_validates(pd):
    N = pd._native
    F = C.c_double()
    box = N.dbl3((10.0, 10.0, 10.0))
    # alpha must be positive; the real-space cutoff x / alpha must stay below half the box
    _expect_einval(pd, "pd_ewald_oracle", 10, 1, box, C.c_double(1.0), C.c_double(0.0), C.c_double(10.0), 7, 1,
                   C.byref(F))
    _expect_einval(pd, "pd_ewald_oracle", 10, 1, box, C.c_double(1.0), C.c_double(0.5), C.c_double(10.0), 1, 1,
                   C.byref(F))
    _expect_einval(pd, "pd_ewald_oracle", 0, 1, box, C.c_double(1.0), C.c_double(0.5), C.c_double(10.0), 2, 1,
                   C.byref(F))
