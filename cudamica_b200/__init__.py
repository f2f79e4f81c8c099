"""B200-native AMICA EM engine (host-side Python mirror of the C-ABI)."""
