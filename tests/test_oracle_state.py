"""The oracle's state setters, used to start it from the GPU's whole state
(positions, velocities, CG warm start, body-contact list with impulses,
particle proxies): copying one oracle cloth's state, in contact with the
sphere, into a fresh one and stepping both gives the same step bit for bit."""
import numpy as np

import bounce_b200 as b3g


def test_state_copy_in_contact_steps_identically(port):
    scene = b3g.sphere_scene(24)
    a = port.PortCloth(scene.mesh, scene.cdef).setup(scene)
    for _ in range(45):
        a.step(scene.dt)
    ca = a.contacts()
    assert ca["active"].sum() > 20  # draped on the sphere
    st = a.state()
    fat = a.describe()["fat_aabb"]
    b = port.PortCloth(scene.mesh, scene.cdef).setup(scene)
    b.set_state(x=st["x"], v=st["v"], dv=st["dv"])
    live = np.nonzero(ca["exists"])[0]
    b.set_contacts(live, np.zeros(live.size, np.uint32), ca["impulses"][live])
    b.set_proxies(fat[:, :3], fat[:, 3:])
    for _ in range(3):
        ia, ib = a.step(scene.dt), b.step(scene.dt)
        assert ia["iterations"] == ib["iterations"] and ia["active_contacts"] == ib["active_contacts"]
        sa, sb = a.state(), b.state()
        assert np.array_equal(sa["x"], sb["x"]) and np.array_equal(sa["v"], sb["v"])
        assert np.array_equal(a.contacts()["impulses"], b.contacts()["impulses"])
