"""Exceptions with the names and meaning of pyPaSWAS/Core/Exceptions.py, so
callers of the reference catch the same types."""


class InvalidOptionException(Exception):
    """Invalid argument or setting (reference: Exceptions.py InvalidOptionException)."""


class HardwareException(Exception):
    """Device missing or unsupported (reference: Exceptions.py HardwareException)."""


class CudaException(Exception):
    """Failure in device code or an invalid result record (reference: Exceptions.py CudaException)."""


class ReaderException(Exception):
    """No sequence data left in an input file (reference: Exceptions.py ReaderException)."""
