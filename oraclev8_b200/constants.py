"""Physical constants of the LH82 step, the exact literals of
oracle_v8/constants.py:25-28 (changing them changes results bit for bit)."""

GRAVITY = 9.81        # m/s^2
R_D = 287.04          # J/(kg K)
C_P = 1004.5          # J/(kg K)
P_REF = 100_000.0     # Pa
