"""alpine_b200: a B200-native (sm_100a) wavefront path tracer behind alpine's API."""
