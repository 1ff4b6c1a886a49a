"""B200-native interval-set AMR hot path (placeholder, filled in below)."""
