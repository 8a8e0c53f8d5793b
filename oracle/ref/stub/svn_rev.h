/* Stand-in for the build-generated revision header. */
#define SVN_REV "oracle"
