import sys
from . import cmake_dir

if "--cmake_dir" in sys.argv:
    print(cmake_dir())
