/* Empty stand-in for the CUDA header that the reference's table headers include;
   the host-side table code they define needs nothing from it. */
