"""B200-native VIA server answer path (drop-in for via-server's Server API)."""
