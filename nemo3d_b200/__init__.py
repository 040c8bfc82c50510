"""B200-native tight-binding eigensolver (package stub)."""
