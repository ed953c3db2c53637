"""SSP-RK3 increment weights of the reference (src/charles/RkWeights.hpp:108-110)."""
ERK3 = [[1.0, 0.0, 0.0], [-0.75, 0.25, 0.0], [-1.0 / 12.0, -1.0 / 12.0, 8.0 / 12.0]]
