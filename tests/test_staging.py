"""Argument checks of the input staging, made before any device work."""

import pytest


def test_prefetch_arguments():
    from frost_b200._lib import FrostError
    from frost_b200.staging import GulpPrefetch
    with pytest.raises(ValueError):
        GulpPrefetch.from_source(lambda b: 0, 1024, 64, depth=1)
    with pytest.raises(ValueError):
        GulpPrefetch.from_source(lambda b: 0, 0, 64)
    with pytest.raises(FrostError):
        GulpPrefetch.from_file("/nonexistent/beam.fil", 0, 1024, 64)
