"""The determinism setting's scoping (ordito/config.py:100-225), on the host."""

from __future__ import annotations

import threading

import ordito_b200 as ob
from ordito_b200 import config


def test_default_override_and_nesting() -> None:
    assert config.is_deterministic() is False
    config.set_deterministic(True)
    try:
        assert ob.is_deterministic() is True
        with config.deterministic(False):
            assert config.is_deterministic() is False
            with config.deterministic(True):
                assert config.is_deterministic() is True
            assert config.is_deterministic() is False
        assert config.is_deterministic() is True
    finally:
        config.set_deterministic(False)
    assert config.is_deterministic() is False


def test_override_is_per_thread_and_restored_on_error() -> None:
    seen = []
    with config.deterministic(True):
        worker = threading.Thread(target=lambda: seen.append(config.is_deterministic()))
        worker.start()
        worker.join()
        assert config.is_deterministic() is True
    assert seen == [False]  # a new thread starts from the process default
    try:
        with config.deterministic(True):
            raise RuntimeError("inside")
    except RuntimeError:
        pass
    assert config.is_deterministic() is False
