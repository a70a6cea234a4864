"""piko-public_b200: Piko's raster and Reyes pipelines on one B200 (placeholder)."""
