"""Copies the reference's own example inputs (the Picacho landslide:
MASTER.dat, the SW .dat, the .top DEM and the .pts source) into this folder,
gzip-compressed, so that tests can run the example without the reference
tree.  Run from the repository root in a container that has the reference:

    python tests/golden/picacho/make_fixture.py

The files are inputs only: the reference ships no expected outputs for them.
"""
import gzip
import os
import shutil

SRC = "/root/reference/EJEMPLOS/Picacho Landslide/Input files"
HERE = os.path.dirname(os.path.abspath(__file__))
FILES = ("Picacho.MASTER.dat", "Picacho.dat", "Picacho.top", "Picacho.pts")


def main():
    for name in FILES:
        with open(os.path.join(SRC, name), "rb") as f, gzip.GzipFile(
                os.path.join(HERE, name + ".gz"), "wb", compresslevel=9, mtime=0) as g:
            shutil.copyfileobj(f, g)


def extract(directory):
    """Writes the example's input files into `directory` (for the tests)."""
    for name in FILES:
        with gzip.open(os.path.join(HERE, name + ".gz"), "rb") as g, open(os.path.join(directory, name), "wb") as f:
            shutil.copyfileobj(g, f)
    return directory


if __name__ == "__main__":
    main()
