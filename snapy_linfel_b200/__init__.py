"""B200-native hydro step for snapy (package root)."""
