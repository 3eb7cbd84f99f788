"""The configuration scenes, built once per test process and shared by the
GPU test files that use them (building the 1,048,576-site mixture's Cech
adjacency takes most of a minute)."""

import functools

from blade_volume_b200 import scenes


@functools.lru_cache(maxsize=None)
def radfoam_ball_262k():
    """262,144 sites in the unit ball, SH 3 (the training benchmark scene)."""
    return scenes.radfoam_ball(262144, seed=0, sh_degree=3)


@functools.lru_cache(maxsize=None)
def powerfoam_1m(bf16: bool):
    """The 1,048,576-site PowerFoam mixture; bf16: SH rounded to BF16 and
    stored as BF16 on the device, else the unrounded FP32 coefficients."""
    m = powerfoam_1m_f32()
    if not bf16:
        return m
    out = m.copy()
    out.sh = scenes.round_to_bf16(m.sh)
    out.sh_bf16 = True
    return out


@functools.lru_cache(maxsize=None)
def powerfoam_1m_f32():
    return scenes.powerfoam_mixture(1048576, seed=0, bf16=False)
