"""B200-native real-time propagation path for SALMON's periodic (ARTED) code."""
