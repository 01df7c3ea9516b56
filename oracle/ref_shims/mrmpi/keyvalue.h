/* Empty stand-in for MapReduce-MPI.  The Vamana build path of the reference
 * never calls it (only the unused BSPWorker transport does); oracle compile
 * only. */
#pragma once
