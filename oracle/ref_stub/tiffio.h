/* Empty stand-in for libtiff's header. The oracle build compiles the reference's
 * CPU filter and noise sources, which include the TIFF IO header transitively but
 * never call libtiff on the whole-stack path (TIFF IO is reached only in resume
 * and disk-block modes, which the oracle does not use). */
