"""B200-native (sm_100a) drop-in for hmfem's pressure solve."""
