"""Run a problem to t_end the way the reference time loop does and collect the
snapshots it would write (src/main.f90:279-292): primitives with THERMAL
pressure, taken after each step that reaches the next output time."""
import numpy as np


def thermal_snapshots(advance, get_prims, t_end, max_steps=100000):
    """advance() takes one step and returns (t, wrote_snapshot);
    get_prims() returns (rho, vx, vy, P_total, Bx, By) numpy arrays."""
    snaps = []
    for _ in range(max_steps):
        t, wrote = advance()
        if wrote:
            rho, vx, vy, P, Bx, By = get_prims()
            snaps.append(dict(t=t, rho=rho, Vx=vx, Vy=vy, P=P - 0.5 * (Bx * Bx + By * By), Bx=Bx, By=By))
        if t >= t_end:
            break
    return snaps


def oracle_snapshots(O, cfg, arrays):
    s = O.State(arrays)

    def advance():
        oc = s.output_count
        O.run(cfg, s, 1)
        return s.t, s.output_count != oc

    return thermal_snapshots(advance, lambda: O.primitives(cfg, s.a), cfg.t_end)


def energy_mean(snap, gamma):
    e = snap["P"] / (gamma - 1.0) + 0.5 * snap["rho"] * (snap["Vx"] ** 2 + snap["Vy"] ** 2) + \
        0.5 * (snap["Bx"] ** 2 + snap["By"] ** 2)
    return float(e.mean())


def mass_drift(snaps):
    """Largest relative change of the total density over the snapshots
    (tests/physics/test_physics.py:46-60)."""
    m0 = snaps[0]["rho"].sum()
    return max(abs(s["rho"].sum() - m0) / m0 for s in snaps)


def field_loop_l1(snaps):
    """Mean |B| change of the advected loop, relative to its mean strength
    (tests/physics/test_physics.py:118-141)."""
    B0 = np.sqrt(snaps[0]["Bx"] ** 2 + snaps[0]["By"] ** 2)
    Bf = np.sqrt(snaps[-1]["Bx"] ** 2 + snaps[-1]["By"] ** 2)
    mean_B0 = B0[B0 > 1e-8].mean() if (B0 > 1e-8).any() else 1.0
    return np.mean(np.abs(Bf - B0)) / mean_B0
