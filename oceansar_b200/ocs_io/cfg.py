"""``.cfg`` parameter files, read and written like ``oceansar/ocs_io/cfg.py:10-198``.

``[section]`` lines open attribute namespaces and ``key=value`` lines become attributes,
converted as the reference converts them: digits -> int, True/False -> bool, ``[...]`` ->
string / bool / float array, anything float() accepts -> float, else the string.  Comments
start with ``#`` or ``;`` (also in-line).  The reference's quirks are kept on purpose so that
every existing ``.cfg`` parses the same way: ``-3`` becomes a float, ``None`` stays the
string 'None', and a one-element array such as ``[0]`` is taken for a section header.
"""
import ast
import re

import numpy as np

_COMMENT = re.compile(r'(^[;#].*$)|(^[\s\t\r\n]*$)')
_SECTION = re.compile(r'\[(\w+)\]')
_VARIABLE = re.compile(r'(\w+)\s*=\s*([\s\w\s\\\:\.,/\'\-\[\]]+)')


class Section(object):
    def __init__(self):
        self.elements = []


def _convert(val):
    if val.isdigit():
        return int(val)
    if val in ('True', 'False'):
        return val == 'True'
    if val[0] == '[':
        if val[1] == '\'':
            return val.replace('\'', '')[1:-1].split(',')
        if val[1] in ('T', 'F'):
            items = val[1:-1].split(',')
            out = np.ones(len(items), dtype=bool)
            for i, it in enumerate(items):
                out[i] = ast.literal_eval(it.strip())
            return out
        return np.array(val[1:-1].split(',')).astype(float)
    try:
        return float(val)
    except ValueError:
        return val


class ConfigFile(object):
    """Parameters of a ``.cfg`` file as ``cfg.<section>.<key>``."""

    def __init__(self, cfg_file_name, str_mode=False):
        self.cfg_file_name = cfg_file_name
        self.str_mode = str_mode
        self.read()

    def read(self):
        self.sections = [self]
        self.elements = []
        current = self
        with open(self.cfg_file_name, 'r') as f:
            for line in f:
                if _COMMENT.search(line):
                    continue
                line = re.sub(r'[;#].*$', '', line.strip())
                m = _SECTION.search(line)
                if m:
                    vars(self)[m.group(1)] = Section()
                    self.sections.append(m.group(1))
                    current = vars(self)[m.group(1)]
                    continue
                m = _VARIABLE.search(line)
                if not m:
                    continue
                key, val = m.group(1), m.group(2)
                vars(current)[key] = val if self.str_mode else _convert(val)
                current.elements.append(key)

    def save(self, alternate_file=None, blank_lines=True):
        with open(alternate_file if alternate_file else self.cfg_file_name, 'w') as f:
            for section in self.sections:
                if section is self:
                    inst = self
                else:
                    f.write('[%s]\n' % section)
                    inst = vars(self)[section]
                for el in inst.elements:
                    v = vars(inst)[el]
                    if type(v) is bool:
                        f.write('%s=%s\n' % (el, 'True' if v else 'False'))
                    elif type(v) is int:
                        f.write('%s=%d\n' % (el, v))
                    elif type(v) in (float, np.float32, np.float64):
                        f.write('%s=%.8f\n' % (el, v))
                    elif type(v) is str:
                        f.write('%s=%s\n' % (el, v))
                    elif type(v) is list:
                        f.write('%s=[' % el + ','.join('\'%s\'' % x for x in v) + ']\n')
                    elif type(v) is np.ndarray:
                        f.write('%s=[' % el + ','.join('%.2f' % x for x in v) + ']\n')
                    else:
                        raise TypeError('Variable type not supported')
                if blank_lines:
                    f.write('\n')
