"""gramsci_b200: B200-native N-point correlation counts (Gramsci's hot path)."""
