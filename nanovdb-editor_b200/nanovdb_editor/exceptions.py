"""Exception types of the reference pymodule (pymodule/nanovdb_editor/exceptions.py)."""


class InvalidArgumentError(ValueError):
    """An argument had the wrong shape, type or value."""


class PipelineError(RuntimeError):
    """The native library reported a failure."""
