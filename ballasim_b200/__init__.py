"""ballasim_b200: a B200-native (sm_100a) implementation of BallaSim's per-pixel event-generation path."""
