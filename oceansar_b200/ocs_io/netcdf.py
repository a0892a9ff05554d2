"""``NETCDFHandler`` (oceansar/ocs_io/netcdf.py): get / set of file variables, with the
``name*`` convention for complex data stored as ``name_r`` / ``name_i``."""
import numpy as np


class NETCDFHandler(object):
    def close(self):
        self.__file__.close()

    def get(self, name):
        if name[-1] == '*':
            re = self.__file__.variables[name[:-1] + '_r'][:]
            content = np.empty(re.shape, dtype=np.complex64)
            content.real = re
            content.imag = self.__file__.variables[name[:-1] + '_i'][:]
            return content
        return self.__file__.variables[name][:]

    def set(self, name, value):
        if name[-1] == '*':
            self.__file__.variables[name[:-1] + '_r'][:] = np.real(value)
            self.__file__.variables[name[:-1] + '_i'][:] = np.imag(value)
        else:
            self.__file__.variables[name][:] = value
