"""B200-native engine for the monodomain hot path of LLNL/Cardioid."""
