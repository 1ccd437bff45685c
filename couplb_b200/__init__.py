"""couplb_b200 -- B200-native (sm_100a) CoupLB LBM + IBM hot path."""
