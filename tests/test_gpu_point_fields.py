"""Point-particle fields for self-gravity and outputs on the GPU against the oracle: the TSC
density and the science fields (FP64 atomics: within 1e-12 of the field's scale), the force
field with its transposed ghost cells and the gathered accelerations (bit-exact), and the
error word for particles the transfers reject."""
import numpy as np
import pytest

from athenak_b200.inputs import make_state
from oracle.oracle import Oracle
from tests.test_point_fields import MESHES, mesh

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def pair(name, t, phys_extra=None):
    from athenak_b200.drag import DeviceDust
    ms = mesh(name)
    st = make_state(ms, [0.1, 0.01], [1.0, 0.5], 2, seed=8, vel_noise=0.05)
    phys = dict(scheme=2, shearing_box=ms.shear_x1, x3_deposit_drop=True)
    phys.update(phys_extra or {})
    o, g = Oracle(st, phys), DeviceDust(st, phys)
    o.set_time(t)
    g.set_time(t)
    return ms, st, o, g


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("t", [0.37, 1.32])
@pytest.mark.parametrize("name", list(MESHES))
def test_gravity_density_force_field_and_gather(name, t):
    ms, st, o, g = pair(name, t)
    rho_o, err = o.point_gravity_density()
    rho_g = g.point_gravity_density().cpu().numpy()
    assert err == 0 and g.error_word() == 0
    assert rel(rho_g, rho_o) < 1e-12
    rng = np.random.default_rng(3)
    owned = np.zeros(ms.field_shape(3))
    ms.active(owned)[...] = rng.standard_normal(ms.active(owned).shape)
    acc_o, err = o.point_gravity_gather(owned)
    acc_g, f_g = g.point_gravity_gather(torch.from_numpy(owned).cuda(), return_field=True)
    assert err == 0 and g.error_word() == 0
    np.testing.assert_array_equal(f_g.cpu().numpy(), o.point_force_field(owned))
    np.testing.assert_array_equal(acc_g.cpu().numpy(), acc_o)


@pytest.mark.parametrize("scheme", [0, 1, 2])
def test_science_fields(scheme):
    ms, st, o, g = pair("shear_x3_outflow", 0.37, dict(scheme=scheme))
    for mass_only, species in ((False, -1), (True, 1), (False, 0)):
        out_o, err = o.point_science_fields(mass_only, species)
        out_g = g.point_science_fields(mass_only, species).cpu().numpy()
        assert err == 0 and g.error_word() == 0
        for v in range(out_o.shape[1]):
            assert rel(out_g[:, v], out_o[:, v]) < 1e-12


def test_rejected_particles_set_the_error_bit():
    from athenak_b200.drag import DeviceDust
    ms = mesh("periodic")
    st = make_state(ms, [0.1], [1.0], 2, seed=8)
    st.pr[16, 5] = -2.0
    st.pr[2, 9] = np.inf
    phys = dict(scheme=2)
    o, g = Oracle(st, phys), DeviceDust(st, phys)
    rho_o, err_o = o.point_gravity_density()
    rho_g = g.point_gravity_density().cpu().numpy()
    assert err_o == 128 and g.error_word() == 128
    assert rel(rho_g, rho_o) < 1e-12
    owned = np.zeros(ms.field_shape(3))
    ms.active(owned)[:, 2] = 1.0
    acc_o, _ = o.point_gravity_gather(owned)
    acc_g = g.point_gravity_gather(torch.from_numpy(owned).cuda()).cpu().numpy()
    np.testing.assert_array_equal(acc_g, acc_o)
    assert np.all(acc_g[:, [5, 9]] == 0.0)
    # the drag's own scheme must be TSC for the gravity transfer
    from athenak_b200 import capi
    g2 = DeviceDust(st, dict(scheme=1))
    with pytest.raises(RuntimeError):
        g2.point_gravity_density()
