"""rkifield_b200 — B200-native SDF ray-march engine for RKIField scenes."""
