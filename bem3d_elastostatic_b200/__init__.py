"""B200-native (sm_100a) boundary-element hot path of QUADESTH."""
