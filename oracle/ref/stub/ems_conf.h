/* Stand-in for the configure-generated ems_conf.h: no optional features. */
