"""Names of the C functions declared in include/*.h."""
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", src, re.M):
            name = m.group(1)
            if name in ("if", "while", "for", "return", "sizeof") or m.group(0).startswith("typedef"):
                continue
            names.append(name)
        # exported data: extern T const *a, *b;
        for m in re.finditer(r"^extern\s+[^;(]*;", src, re.M):
            names.extend(re.findall(r"\*\s*([A-Za-z_]\w*)", m.group(0)))
    return names
