/*
 * Stand-in for the reference's logwrite() (sourceCode/log/log.c:12-29), used
 * only when linking the reference ICON-GPU sources into oracle/_ref/.  The
 * reference appends to a path read from an install-time config file and does
 * nothing when that file is absent; this stub always does nothing.
 * TEST INFRASTRUCTURE ONLY.
 */
int logwrite(char *loginfo)
{
    (void)loginfo;
    return 0;
}
