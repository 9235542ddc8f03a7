"""B200-native engine for fly-in-silico's whole-brain LIF step."""
