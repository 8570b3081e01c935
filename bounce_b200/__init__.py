"""B200-native implicit cloth step for Bounce (placeholder)."""
