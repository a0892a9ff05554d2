"""Oracle (test infrastructure only): ``.cfg`` reader restating ``oceansar/ocs_io/cfg.py:67-143``.

Sections become attribute namespaces; values convert to int (``isdigit``), bool,
string / bool / float arrays, float, else string.  A one-element array such as ``[0]``
matches the section pattern first, exactly as in the reference.
"""
import ast
import re

import numpy as np


class Section:
    def __init__(self):
        self.elements = []


class ConfigFile:
    def __init__(self, cfg_file_name):
        self.sections = [self]
        self.elements = []
        cur = self
        with open(cfg_file_name) as f:
            for line in f:
                if re.search(r'(^[;#].*$)|(^[\s\t\r\n]*$)', line):
                    continue
                line = line.rstrip().lstrip()
                line = re.sub(r'[;#].*$', '', line)
                s = re.search(r'\[(\w+)\]', line)
                if s:
                    vars(self)[s.group(1)] = Section()
                    self.sections.append(s.group(1))
                    cur = vars(self)[s.group(1)]
                    continue
                s = re.search(r'(\w+)\s*=\s*([\s\w\s\\\:\.,/\'\-\[\]]+)', line)
                if not s:
                    continue
                key, val = s.group(1), s.group(2)
                if val.isdigit():
                    v = int(val)
                elif val in ('True', 'False'):
                    v = val == 'True'
                elif val[0] == '[':
                    if val[1] == '\'':
                        v = val.replace('\'', '')[1:-1].split(',')
                    elif val[1] in ('T', 'F'):
                        tmp = val[1:-1].split(',')
                        v = np.ones(len(tmp), dtype=bool)
                        for i, t in enumerate(tmp):
                            v[i] = ast.literal_eval(t.strip())
                    else:
                        v = np.array(val[1:-1].split(',')).astype(float)
                else:
                    try:
                        v = float(val)
                    except ValueError:
                        v = val
                vars(cur)[key] = v
                cur.elements.append(key)
