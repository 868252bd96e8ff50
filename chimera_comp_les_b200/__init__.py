"""B200-native compressible RHS + SSP-RK stage update (placeholder; filled in below)."""
