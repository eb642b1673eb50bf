"""B200-native implementation of CasPhy's tree-building hot path."""
