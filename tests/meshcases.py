"""Mesh configurations shared by the tests (INI text with reference keys)."""
from kratos_polrad_b200.mesh import MeshConfig, RefineRegion

# Slab of the plain-forward configuration: 128x128x64 cells in 16^3 blocks,
# periodic in x and y.
SLAB = MeshConfig((0, 0, 0), (128, 128, 64), (128, 128, 64), (16, 16, 16),
                  (True, True, False))

# Small AMR meshes: one refined box, periodic and not.
AMR_BOX = MeshConfig((0, 0, 0), (1, 1, 1), (64, 64, 64), (16, 16, 16), (False,) * 3,
                     [RefineRegion(1, (0.375, 0.375, 0.375), (0.625, 0.625, 0.625))])
AMR_PERIODIC = MeshConfig((-1, -2, 0.5), (1, 2, 2.5), (64, 64, 32), (8, 8, 8),
                          (True, False, True),
                          [RefineRegion(1, (-1.0, -2.0, 0.5), (-0.75, -1.5, 0.75)),
                           RefineRegion(2, (0.25, 0.5, 1.5), (0.3, 0.6, 1.6))])
THREE_LEVEL = MeshConfig((0, 0, 0), (2, 2, 2), (64, 64, 64), (8, 8, 8), (True, True, True),
                         [RefineRegion(2, (0.9, 0.9, 0.9), (1.1, 1.1, 1.1)),
                          RefineRegion(1, (0.1, 1.6, 0.2), (0.2, 1.9, 0.3))])

CASES = {"slab": SLAB, "amr_box": AMR_BOX, "amr_periodic": AMR_PERIODIC,
         "three_level": THREE_LEVEL}
