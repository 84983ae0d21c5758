"""Python host side of the PFSF B200 solve: ctypes binding of libpfsf.so,
seeded synthetic island generators and a torch wrapper."""
from . import capi, synth  # noqa: F401

__all__ = ["capi", "synth"]
