"""voxarmps_b200 -- Blackwell-native MPS solver core (sm_100a)."""
