"""B200-native GF2 Kadanoff-Baym hot path (density-fitted / full-U second-Born
self-energy, Dyson time step, Legendre mixed-component convolutions,
predictor) behind a C ABI (include/nedy.h)."""
