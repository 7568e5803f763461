"""B200-native Smith-Waterman engine with pyPaSWAS's driver interface."""
