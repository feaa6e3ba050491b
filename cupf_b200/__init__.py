"""B200-native 3D APT multi-grain phase-field step (cuPF hot path)."""
