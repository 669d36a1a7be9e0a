// Empty stand-in: the host ingest compiled for the oracle needs nothing from this header.
#pragma once
