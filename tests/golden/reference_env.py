"""The reference loader of oracle/reference_env.py, under the name the
golden-fixture script and the tests import."""

from oracle.reference_env import (  # noqa: F401
    REFERENCE_ROOT,
    REPO,
    SOURCE_ROOT,
    STAGED_ROOT,
    load_reference,
    reference_available,
    source_available,
)
