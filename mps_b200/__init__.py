"""B200-native MPS time-step hot path (see DESIGN.md at the repository root)."""
