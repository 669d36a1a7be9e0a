// Empty stand-in: no device instantiations in the host build.
