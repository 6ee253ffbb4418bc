"""Exception types named after the Julia exceptions the reference throws, so callers and tests
can match on the same names and message substrings."""


class ArgumentError(ValueError):
    """An invalid argument (Julia's ArgumentError)."""


class DimensionMismatch(ValueError):
    """Arrays whose sizes disagree (Julia's DimensionMismatch)."""
