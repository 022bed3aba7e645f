"""B200-native periodic method-of-moments fill-and-solve for PSSFSS-style analyses."""
