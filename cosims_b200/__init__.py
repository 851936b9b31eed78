"""B200-native trajectory-method collision cross-section (CCS) engine."""
