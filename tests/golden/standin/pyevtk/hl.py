"""Stand-in for ``pyevtk.hl``: the fixture generator writes no VTK (test infrastructure only)."""


def gridToVTK(*args, **kwargs):
    raise NotImplementedError("stand-in: VTK export is not used by the fixture generator")
