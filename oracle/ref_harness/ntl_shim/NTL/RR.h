// Empty stand-in: kunpBFV includes <NTL/RR.h> but uses no RR type on its BFV path.
#pragma once
