"""B200-native iTPS CTMRG environment (drop-in for TeNeS's CTMRG path)."""
