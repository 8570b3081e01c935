"""A scripted sequence of particle edits between steps (b3Particle API,
include/bounce/cloth/particle.h:63-111): forces, translations, velocities,
positions and type changes among static, kinematic and dynamic, several on
one particle in the same step.  Shared by the CPU and GPU parity tests."""
import numpy as np

STATIC, KINEMATIC, DYNAMIC = 0, 1, 2


def edits(step: int, n: int):
    """The edits before `step`, in order: (op, vertex, argument)."""
    a, b, c, d = n // 3, n // 2, (2 * n) // 3, n - 7
    script = {
        3: [("apply_force", a, (0.0, 4.0, 0.0)), ("apply_translation", b, (0.01, 0.0, -0.005)),
            ("set_velocity", c, (0.0, 1.0, 0.5))],
        6: [("set_type", a, STATIC), ("set_position", a, None), ("apply_force", a, (0.0, 9.0, 0.0))],
        9: [("set_type", b, KINEMATIC), ("set_velocity", b, (0.0, 0.3, 0.0)), ("apply_force", b, (1.0, 0.0, 0.0))],
        12: [("set_type", a, DYNAMIC), ("set_velocity", d, (0.2, 0.0, 0.0)), ("apply_translation", d, (0.0, 0.02, 0.0)),
             ("apply_translation", d, (0.0, 0.0, 0.01))],
        15: [("set_type", b, DYNAMIC), ("set_type", c, STATIC), ("set_type", c, DYNAMIC)],
        18: [("set_position", d, None), ("set_velocity", d, (0.0, -0.5, 0.0))],
    }
    return script.get(step, [])


def apply(cloth, step: int, positions: np.ndarray, gpu: bool):
    """Apply the edits of `step` through either API (`positions`: the current
    positions, for the set_position targets)."""
    for op, v, arg in edits(step, positions.shape[0]):
        if op == "set_position":
            arg = positions[v] + np.array([0.0, 0.05, 0.02], np.float32)
        if gpu:
            p = cloth.particle(v)
            getattr(p, op)(arg)
        else:
            getattr(cloth, op)(v, arg)
