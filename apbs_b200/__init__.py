"""apbs_b200: B200-native (sm_100a) finite-difference PMG Poisson-Boltzmann solver."""
