"""tsb: B200-native TorchSim classical-potential hot path (placeholder during bring-up)."""
