#!/bin/sh
# Copies the reference's two shipped graphs (dataset/*.bin) into datasets/
# (git-ignored; travels with the working tree to a GPU box).  The files are
# inputs, not fixtures: the golden counts come from the reference README.
set -e
SRC=${1:-/root/reference/dataset}
DST=$(dirname "$0")/../../datasets
mkdir -p "$DST"
cp "$SRC"/soc-epinions.bin "$SRC"/email-euall.bin "$DST"/
