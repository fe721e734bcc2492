"""Logging for the OP2 host layer (pyop2/logger.py:39-53)."""

import logging

logger = logging.getLogger('pyop2')
_ch = logging.StreamHandler()
_ch.setFormatter(logging.Formatter('%(name)s:%(levelname)s %(message)s'))
logger.addHandler(_ch)

debug = logger.debug
info = logger.info
warning = logger.warning
error = logger.error
critical = logger.critical


def set_log_level(level):
    if isinstance(level, str) and level == 'WARN':
        level = 'WARNING'
    logger.setLevel(level)
