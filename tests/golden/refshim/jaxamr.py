"""Empty stand-in for the external ``jaxamr`` package (AMR is not exercised)."""


class amr:  # noqa: N801
    pass
