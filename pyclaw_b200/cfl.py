"""CFL holder (src/pyclaw/cfl.py:5-25).  On the device path the value is the
CFL number the step kernel's last block reduced for the last step."""


class CFL(object):
    def __init__(self, global_max):
        self._global_max = global_max

    def get_global_max(self):
        return self._global_max

    def get_cached_max(self):
        return self._global_max

    def set_local_max(self, new_local_max):
        self._global_max = new_local_max

    def update_global_max(self, new_local_max):
        self._global_max = new_local_max
