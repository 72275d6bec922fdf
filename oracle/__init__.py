"""Oracle for the world DEM step: a CPU restatement of the reference's algorithm
(dem_oracle.c) and the build recipe for the reference's own step (build.py).
Test infrastructure only; the product (world_b200/) never imports it."""
