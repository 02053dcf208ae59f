"""Placeholder for ``xarray`` so that the reference's I/O modules import; any use raises."""


def __getattr__(name):
    raise ImportError("xarray is not available; the I/O path is not exercised by the golden generator")
