"""B200-native dyphur frame step."""
