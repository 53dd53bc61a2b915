from .geom import suggest_volume_extent  # noqa: F401
