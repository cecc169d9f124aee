"""B200-native SPH hot path (see include/uph.h for the C ABI)."""
