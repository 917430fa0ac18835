#!/bin/sh
# Copies the reference's two shipped graphs (dataset/*.bin) into datasets/
# (git-ignored; travels with the working tree to a GPU box).  The files are
# inputs, not fixtures: the golden counts come from the reference README.
# Usage: fetch_datasets.sh <reference>/dataset
set -e
if [ -z "$1" ]; then echo "usage: $0 <reference project>/dataset" >&2; exit 1; fi
SRC=$1
DST=$(dirname "$0")/../../datasets
mkdir -p "$DST"
cp "$SRC"/soc-epinions.bin "$SRC"/email-euall.bin "$DST"/
