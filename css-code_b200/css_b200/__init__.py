"""css_b200: B200 (sm_100a) implementation of the CSS time-step hot path."""
from .params import CssParams, default_params  # noqa: F401
