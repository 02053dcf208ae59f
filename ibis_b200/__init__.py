"""B200-native hourly land-surface step of IBIS 3.0 (see README.md)."""
