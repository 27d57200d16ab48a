"""B200-native lattice Boltzmann wind-tunnel compute path."""
