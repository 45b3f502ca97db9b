"""Stand-in for ``ruamel.yaml``: the fixture generator reads no YAML (test infrastructure only)."""


class YAML:
    def __init__(self, *args, **kwargs):
        raise NotImplementedError("stand-in: YAML is not used by the fixture generator")
