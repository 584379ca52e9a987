"""CPU oracle of the explicit 2D FEM step -- TEST INFRASTRUCTURE ONLY.

Restates the reference's (FlatWorld) algorithm on the CPU: fw_oracle.c for the
device kernels (FP32 / FP32-with-FMA / FP64 builds) and scene.py for the
host-side construction and stepping logic.  Only tests/, __graft_entry__.smoke()
and bench.py's CPU legs use it, as the checker; the product (flatworld_b200)
never imports it.
"""

from .scene import OracleLoop, boundary_nodes_literal, char_length_literal, point_stress  # noqa: F401
