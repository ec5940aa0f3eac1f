"""The reference's known-answer tests (tests/tests.cpp, tests/audit_tests.cpp) on the CUDA path."""
import pytest

import known_answers
from gpu_impl import GpuImpl

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", known_answers.ALL, ids=lambda f: f.__name__)
def test_known_answers_on_gpu(case):
    case(GpuImpl())
