"""B200-native PUReIBM-PS2D-FD1D time-step engine (host side)."""
