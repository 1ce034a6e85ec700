def colored(text, *_, **__):
    return text
