/* Empty revision header: qmcpack_version.cpp includes it, and an empty one
 * is what the reference's build writes outside a git checkout. */
